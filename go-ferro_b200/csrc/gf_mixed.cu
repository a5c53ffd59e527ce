// Mixed-precision (FP32) stage sequence of the engine, in a translation unit
// of its own so that it is compiled with FMA contraction: gf_engine.cu is
// compiled with -fmad=false because the FP64 parity kernels must round every
// multiply and add separately, as the reference's host build does; the FP32
// kernels have no such constraint and are instruction-bound, so fused
// multiply-adds shorten them.  This file instantiates only the <S, float>
// stage kernels and exports gf_mixed_enqueue_step / gf_mixed_elastic_setup,
// declared in gf_engine.cu.
#define GF_MIXED_TU 1
#include "gf_engine.cu"
