// ryser_dense_sdd_inst.cu -- split-dd dense Ryser kernels (certified bound for
// real matrices), orders 4..40.
#include "ryser_dense_sdd.cuh"

namespace perm {
#define PERM_SDD_CASE(n) \
  case n: return reinterpret_cast<const void*>(&ryser_dense_sdd_kernel<n>);
const void* dense_sdd_kernel(int n) {
  switch (n) {
    PERM_SDD_CASE(4) PERM_SDD_CASE(5) PERM_SDD_CASE(6) PERM_SDD_CASE(7) PERM_SDD_CASE(8) PERM_SDD_CASE(9)
    PERM_SDD_CASE(10) PERM_SDD_CASE(11) PERM_SDD_CASE(12) PERM_SDD_CASE(13) PERM_SDD_CASE(14)
    PERM_SDD_CASE(15) PERM_SDD_CASE(16) PERM_SDD_CASE(17) PERM_SDD_CASE(18) PERM_SDD_CASE(19)
    PERM_SDD_CASE(20) PERM_SDD_CASE(21) PERM_SDD_CASE(22) PERM_SDD_CASE(23) PERM_SDD_CASE(24)
    PERM_SDD_CASE(25) PERM_SDD_CASE(26) PERM_SDD_CASE(27) PERM_SDD_CASE(28) PERM_SDD_CASE(29)
    PERM_SDD_CASE(30) PERM_SDD_CASE(31) PERM_SDD_CASE(32) PERM_SDD_CASE(33) PERM_SDD_CASE(34)
    PERM_SDD_CASE(35) PERM_SDD_CASE(36) PERM_SDD_CASE(37) PERM_SDD_CASE(38) PERM_SDD_CASE(39)
    PERM_SDD_CASE(40)
    default: return nullptr;
  }
}
#undef PERM_SDD_CASE
}  // namespace perm
