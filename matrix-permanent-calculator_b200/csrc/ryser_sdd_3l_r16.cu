// ryser_sdd_3l_r16.cu -- three-level split-dd Ryser kernels whose columns 1
// and 2 touch rows 0..15 only and column 0 rows 0..R1-1 (R1 in 8, 12), orders
// 24..40, 3 CTAs per SM.
#include "ryser_dense_sdd.cuh"

namespace perm {
const void* sdd_3l_kernel_r16(int n, int r1) {
  switch (n) {
    case 24:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<24, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<24, 12, 16, 3>);
      return nullptr;
    case 25:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<25, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<25, 12, 16, 3>);
      return nullptr;
    case 26:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<26, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<26, 12, 16, 3>);
      return nullptr;
    case 27:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<27, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<27, 12, 16, 3>);
      return nullptr;
    case 28:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<28, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<28, 12, 16, 3>);
      return nullptr;
    case 29:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<29, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<29, 12, 16, 3>);
      return nullptr;
    case 30:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<30, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<30, 12, 16, 3>);
      return nullptr;
    case 31:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<31, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<31, 12, 16, 3>);
      return nullptr;
    case 32:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<32, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<32, 12, 16, 3>);
      return nullptr;
    case 33:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<33, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<33, 12, 16, 3>);
      return nullptr;
    case 34:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<34, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<34, 12, 16, 3>);
      return nullptr;
    case 35:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<35, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<35, 12, 16, 3>);
      return nullptr;
    case 36:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<36, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<36, 12, 16, 3>);
      return nullptr;
    case 37:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<37, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<37, 12, 16, 3>);
      return nullptr;
    case 38:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<38, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<38, 12, 16, 3>);
      return nullptr;
    case 39:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<39, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<39, 12, 16, 3>);
      return nullptr;
    case 40:
      if (r1 == 8) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<40, 8, 16, 3>);
      if (r1 == 12) return reinterpret_cast<const void*>(&ryser_sdd_3l_kernel<40, 12, 16, 3>);
      return nullptr;
    default:
      return nullptr;
  }
}
}  // namespace perm
