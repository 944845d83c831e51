// ryser_sdd_3l_r20.cu -- three-level split-dd Ryser kernels whose columns 1
// and 2 touch rows 0..19 only and column 0 rows 0..R1-1 (R1 in 8, 12, 16),
// orders 24..40, 3 CTAs per SM (2 for order/R1 31/8, 35/8, 39/8, which spill
// at 3).
#include "ryser_dense_sdd.cuh"

namespace perm {
const void* sdd_3l_kernel_r20(int n, int r1) {
  switch (n) {
    case 24:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<24, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<24, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<24, 16, 20, 3>);
      return nullptr;
    case 25:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<25, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<25, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<25, 16, 20, 3>);
      return nullptr;
    case 26:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<26, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<26, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<26, 16, 20, 3>);
      return nullptr;
    case 27:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<27, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<27, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<27, 16, 20, 3>);
      return nullptr;
    case 28:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<28, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<28, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<28, 16, 20, 3>);
      return nullptr;
    case 29:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<29, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<29, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<29, 16, 20, 3>);
      return nullptr;
    case 30:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<30, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<30, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<30, 16, 20, 3>);
      return nullptr;
    case 31:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<31, 8, 20, 2>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<31, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<31, 16, 20, 3>);
      return nullptr;
    case 32:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<32, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<32, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<32, 16, 20, 3>);
      return nullptr;
    case 33:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<33, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<33, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<33, 16, 20, 3>);
      return nullptr;
    case 34:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<34, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<34, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<34, 16, 20, 3>);
      return nullptr;
    case 35:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<35, 8, 20, 2>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<35, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<35, 16, 20, 3>);
      return nullptr;
    case 36:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<36, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<36, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<36, 16, 20, 3>);
      return nullptr;
    case 37:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<37, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<37, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<37, 16, 20, 3>);
      return nullptr;
    case 38:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<38, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<38, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<38, 16, 20, 3>);
      return nullptr;
    case 39:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<39, 8, 20, 2>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<39, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<39, 16, 20, 3>);
      return nullptr;
    case 40:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<40, 8, 20, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<40, 12, 20, 3>);
      if (r1 == 16) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<40, 16, 20, 3>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
