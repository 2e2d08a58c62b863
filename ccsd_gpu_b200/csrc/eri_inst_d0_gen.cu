// ERI kernel launchers for derivative order 0, shells up to l = 4.
#include "eri_kernels.cuh"

namespace cb {
CB_ERI_INSTANTIATE(0, false)
}  // namespace cb
