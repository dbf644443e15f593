/* Project-written stand-in for MATLAB's matrix.h: everything lives in mex.h. */
#include "mex.h"
