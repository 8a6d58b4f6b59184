/* ippvm.h -- oracle stand-in; every declaration lives in ipps.h. */
#include "ipps.h"
