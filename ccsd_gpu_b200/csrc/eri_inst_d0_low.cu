// ERI kernel launchers for derivative order 0, every shell l <= 2 (compile-time recurrences).
#include "eri_kernels.cuh"

namespace cb {
CB_ERI_INSTANTIATE(0, true)
}  // namespace cb
