// Force-included before the reference's host sources (g++ -include): the MSVC extensions they use
// -- std::exception(const char *), strcpy_s -- mapped onto standard C++.  Every standard header
// the sources include is pulled in first so that the exception alias below reaches only the
// reference's own code.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <sys/types.h>
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

namespace std {
struct ref_shim_exception : public exception {
    std::string msg;
    ref_shim_exception(const char *m = "") : msg(m ? m : "") {}
    const char *what() const noexcept override { return msg.c_str(); }
};
}  // namespace std
#define exception ref_shim_exception
#define strcpy_s(dst, src) strcpy(dst, src)
namespace stdext {}   // MSVC's extension namespace, named by a using-directive in LabelingAlgs.hpp
