// cb_fp64.cu -- FP64 instantiation of the phase kernels.  Compiled with
// -fmad=false so no multiply-add is contracted: every expression rounds
// exactly as the reference serial model's does (bit parity).
#include "cb_ops_impl.cuh"

template struct cb::Ops<double>;

#include "cb_batch_impl.cuh"
template struct cb::BatchOps<double>;
