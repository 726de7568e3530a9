// Test infrastructure only: exposes, with C linkage, the functions of the
// reference's MultiQW.cpp that compile without Eigen or ApproxTools — the bit
// helpers (MultiQW.cpp:16-34), the inverse normal my_normcdfinvf
// (MultiQW.cpp:39-86) and the AVX-512 hot loop Clenshaw_step
// (MultiQW.cpp:88-173). The build recipe (oracle/Makefile, target `ref`)
// extracts exactly that span from the reference source into
// oracle/_ref/ref_span.inc; nothing of it is committed. The Eigen-dependent
// driver (Clenshaw, main) is not buildable here because Eigen 3.4 and the
// ApproxTools submodule are absent; its loop is restated in mqw_oracle.cpp
// instead.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "vcl2/vectorclass.h"

#include "ref_span.inc"

extern "C" {

float ref_my_normcdfinvf(float a) { return my_normcdfinvf(a); }

unsigned ref_gray(unsigned v) { return grey(v); }

unsigned ref_log2_of_lsb(int v) { return log2(LSB(v)); }

void ref_clenshaw_step(float* b1, float* b2, float* hp, float* psi, unsigned n,
                       float scale, float gamma, float coef) {
  Clenshaw_step(b1, b2, hp, psi, n, scale, gamma, coef);
}

}  // extern "C"
