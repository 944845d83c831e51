// ryser_dense_tc_g4.cu -- tensor-core dense Ryser kernels (kind::i8 row sums) with
// product groups of 4 rows, orders 16..64.
#include "ryser_dense_tc.cuh"

namespace perm {
const void* dense_tc_kernel_g4(int n) {
  switch (n) {
    case 16: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<16, 4>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<17, 4>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<18, 4>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<19, 4>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<20, 4>);
    case 21: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<21, 4>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<22, 4>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<23, 4>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<24, 4>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<25, 4>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<26, 4>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<27, 4>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<28, 4>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<29, 4>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<30, 4>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<31, 4>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<32, 4>);
    case 33: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<33, 4>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<34, 4>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<35, 4>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<36, 4>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<37, 4>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<38, 4>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<39, 4>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<40, 4>);
    case 41: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<41, 4>);
    case 42: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<42, 4>);
    case 43: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<43, 4>);
    case 44: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<44, 4>);
    case 45: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<45, 4>);
    case 46: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<46, 4>);
    case 47: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<47, 4>);
    case 48: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<48, 4>);
    case 49: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<49, 4>);
    case 50: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<50, 4>);
    case 51: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<51, 4>);
    case 52: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<52, 4>);
    case 53: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<53, 4>);
    case 54: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<54, 4>);
    case 55: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<55, 4>);
    case 56: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<56, 4>);
    case 57: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<57, 4>);
    case 58: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<58, 4>);
    case 59: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<59, 4>);
    case 60: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<60, 4>);
    case 61: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<61, 4>);
    case 62: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<62, 4>);
    case 63: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<63, 4>);
    case 64: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<64, 4>);
    default: return nullptr;
  }
}
}  // namespace perm
