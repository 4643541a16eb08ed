// Test infrastructure only. Linked into the second oracle build, libtwofold_ref_rounded.so, where it binds
// the reference's float calls to sinf, cosf, atan2f and asinf (continuous collision turns sweeps with them)
// to correctly rounded values: the double function rounded to float. The reference's own sources are
// unchanged; only the platform library it calls differs. Against this build the B200 library's continuous
// pass is compared bit for bit; against the plain build, which calls the host's float functions, it can
// differ by an ulp wherever those round the other way.
#include <cmath>

extern "C" {
float sinf(float x) { return (float)std::sin((double)x); }
float cosf(float x) { return (float)std::cos((double)x); }
float atan2f(float y, float x) { return (float)std::atan2((double)y, (double)x); }
float asinf(float x) { return (float)std::asin((double)x); }
}
