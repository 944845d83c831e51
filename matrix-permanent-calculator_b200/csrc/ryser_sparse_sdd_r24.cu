// ryser_sparse_sdd_r24.cu -- sparse-layout split-dd Ryser kernels whose
// columns 0..2 touch rows 0..23 only, orders 28..40: the rolled step loop,
// 3 CTAs per SM (inner rows in registers, the others in shared memory); 2
// at orders 31, 35 and 39, which spill at 3.
#include "ryser_dense_sdd.cuh"

namespace perm {
#define PERM_SPSDD_CASE(n) \
  case n: return reinterpret_cast<const void*>(&ryser_sparse_sdd_kernel<n, 24, 3, true>);
#define PERM_SPSDD_CASE2(n) \
  case n: return reinterpret_cast<const void*>(&ryser_sparse_sdd_kernel<n, 24, 2, true>);
const void* sparse_sdd_kernel_r24(int n) {
  switch (n) {
    PERM_SPSDD_CASE(28) PERM_SPSDD_CASE(29) PERM_SPSDD_CASE(30) PERM_SPSDD_CASE2(31) PERM_SPSDD_CASE(32)
    PERM_SPSDD_CASE(33) PERM_SPSDD_CASE(34) PERM_SPSDD_CASE2(35) PERM_SPSDD_CASE(36) PERM_SPSDD_CASE(37)
    PERM_SPSDD_CASE(38) PERM_SPSDD_CASE2(39) PERM_SPSDD_CASE(40)
    default: return nullptr;
  }
}
#undef PERM_SPSDD_CASE
#undef PERM_SPSDD_CASE2
}  // namespace perm
