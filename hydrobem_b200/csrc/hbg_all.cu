// hbg_all.cu -- the main translation unit of libhydrobem_gpu.so (hbg_statics.cu is the other one,
// compiled without floating-point contraction).
#include "hbg_freq.cu"
#include "hbg_motion.cu"
#include "hbg_kochin.cu"
#include "hbg_lu.cu"
#include "hbg_mixed.cu"
#include "hbg_peaks.cu"
#include "hbg_surrogate.cu"
#include "hbg_api.cu"
#include "hbg_gdf.cu"
#include "hbg_model.cu"
#include "hbg_noalloc.cu"
