// ERI kernel launchers for derivative order 1, every shell l <= 2 (compile-time recurrences).
#include "eri_kernels.cuh"

namespace cb {
CB_ERI_INSTANTIATE(1, true)
}  // namespace cb
