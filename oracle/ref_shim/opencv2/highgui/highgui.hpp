// Empty stand-in for <opencv2/highgui/highgui.hpp> (nothing of it is used by the CPU labelers).
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "../core/core.hpp"
