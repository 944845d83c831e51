// ryser_dense_tc_g6.cu -- tensor-core dense Ryser kernels (kind::i8 row sums) with
// product groups of 6 rows, orders 16..64.
#include "ryser_dense_tc.cuh"

namespace perm {
const void* dense_tc_kernel_g6(int n) {
  switch (n) {
    case 16: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<16, 6>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<17, 6>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<18, 6>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<19, 6>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<20, 6>);
    case 21: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<21, 6>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<22, 6>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<23, 6>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<24, 6>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<25, 6>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<26, 6>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<27, 6>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<28, 6>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<29, 6>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<30, 6>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<31, 6>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<32, 6>);
    case 33: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<33, 6>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<34, 6>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<35, 6>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<36, 6>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<37, 6>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<38, 6>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<39, 6>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<40, 6>);
    case 41: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<41, 6>);
    case 42: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<42, 6>);
    case 43: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<43, 6>);
    case 44: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<44, 6>);
    case 45: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<45, 6>);
    case 46: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<46, 6>);
    case 47: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<47, 6>);
    case 48: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<48, 6>);
    case 49: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<49, 6>);
    case 50: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<50, 6>);
    case 51: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<51, 6>);
    case 52: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<52, 6>);
    case 53: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<53, 6>);
    case 54: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<54, 6>);
    case 55: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<55, 6>);
    case 56: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<56, 6>);
    case 57: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<57, 6>);
    case 58: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<58, 6>);
    case 59: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<59, 6>);
    case 60: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<60, 6>);
    case 61: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<61, 6>);
    case 62: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<62, 6>);
    case 63: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<63, 6>);
    case 64: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<64, 6>);
    default: return nullptr;
  }
}
}  // namespace perm
