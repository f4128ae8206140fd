// hbg_all.cu -- the single translation unit of libhydrobem_gpu.so (the __constant__ tables and
// Gauss nodes are defined once and seen by every kernel).
#include "hbg_statics.cu"
#include "hbg_freq.cu"
#include "hbg_lu.cu"
#include "hbg_mixed.cu"
#include "hbg_api.cu"
#include "hbg_model.cu"
