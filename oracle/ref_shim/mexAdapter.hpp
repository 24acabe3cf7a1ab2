// TEST INFRASTRUCTURE ONLY -- stand-in for MATLAB's mexAdapter.hpp.  In MATLAB it
// supplies the C entry point that instantiates the file's MexFunction; here
// oracle/ref_entry.cpp does that after including the reference source.
#pragma once
#include "mex.hpp"
