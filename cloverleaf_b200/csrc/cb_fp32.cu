// cb_fp32.cu -- FP32 instantiation of the phase kernels (the FP32 storage
// form; FP64 where the kernels say `double`).  Multiply-adds may contract.
#include "cb_ops_impl.cuh"

template struct cb::Ops<float>;

#include "cb_batch_impl.cuh"
template struct cb::BatchOps<float>;
