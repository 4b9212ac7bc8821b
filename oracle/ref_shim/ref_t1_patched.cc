// ref_t1_patched.cc -- C++ build of ref_t1.c against the patched copy of
// coefficient_coder.cl (state helpers take their register by reference,
// defects D1/D2 fixed).  TEST INFRASTRUCTURE ONLY.
extern "C" {
#include "ref_t1.c"
}
