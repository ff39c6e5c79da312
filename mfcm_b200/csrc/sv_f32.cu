// sv_f32.cu -- FP32 instantiation of the stage kernels (multiply-add contraction allowed).
#define SV_T float
#include "sv_inst.cuh"
