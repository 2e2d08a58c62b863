// ERI kernel launchers for derivative order 1, shells up to l = 4.
#include "eri_kernels.cuh"

namespace cb {
CB_ERI_INSTANTIATE(1, false)
}  // namespace cb
