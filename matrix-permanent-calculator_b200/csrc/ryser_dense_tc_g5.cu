// ryser_dense_tc_g5.cu -- tensor-core dense Ryser kernels (kind::i8 row sums) with
// product groups of 5 rows, orders 16..64.
#include "ryser_dense_tc.cuh"

namespace perm {
const void* dense_tc_kernel_g5(int n) {
  switch (n) {
    case 16: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<16, 5>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<17, 5>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<18, 5>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<19, 5>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<20, 5>);
    case 21: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<21, 5>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<22, 5>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<23, 5>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<24, 5>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<25, 5>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<26, 5>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<27, 5>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<28, 5>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<29, 5>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<30, 5>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<31, 5>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<32, 5>);
    case 33: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<33, 5>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<34, 5>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<35, 5>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<36, 5>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<37, 5>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<38, 5>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<39, 5>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<40, 5>);
    case 41: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<41, 5>);
    case 42: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<42, 5>);
    case 43: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<43, 5>);
    case 44: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<44, 5>);
    case 45: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<45, 5>);
    case 46: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<46, 5>);
    case 47: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<47, 5>);
    case 48: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<48, 5>);
    case 49: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<49, 5>);
    case 50: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<50, 5>);
    case 51: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<51, 5>);
    case 52: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<52, 5>);
    case 53: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<53, 5>);
    case 54: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<54, 5>);
    case 55: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<55, 5>);
    case 56: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<56, 5>);
    case 57: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<57, 5>);
    case 58: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<58, 5>);
    case 59: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<59, 5>);
    case 60: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<60, 5>);
    case 61: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<61, 5>);
    case 62: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<62, 5>);
    case 63: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<63, 5>);
    case 64: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<64, 5>);
    default: return nullptr;
  }
}
}  // namespace perm
