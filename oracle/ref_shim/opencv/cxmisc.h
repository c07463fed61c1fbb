// empty stand-in for <opencv/cxmisc.h> (test infrastructure only)
