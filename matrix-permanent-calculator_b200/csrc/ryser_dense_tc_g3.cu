// ryser_dense_tc_g3.cu -- tensor-core dense Ryser kernels (kind::i8 row sums) with
// product groups of 3 rows, orders 16..64.
#include "ryser_dense_tc.cuh"

namespace perm {
const void* dense_tc_kernel_g3(int n) {
  switch (n) {
    case 16: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<16, 3>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<17, 3>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<18, 3>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<19, 3>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<20, 3>);
    case 21: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<21, 3>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<22, 3>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<23, 3>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<24, 3>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<25, 3>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<26, 3>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<27, 3>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<28, 3>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<29, 3>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<30, 3>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<31, 3>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<32, 3>);
    case 33: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<33, 3>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<34, 3>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<35, 3>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<36, 3>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<37, 3>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<38, 3>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<39, 3>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<40, 3>);
    case 41: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<41, 3>);
    case 42: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<42, 3>);
    case 43: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<43, 3>);
    case 44: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<44, 3>);
    case 45: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<45, 3>);
    case 46: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<46, 3>);
    case 47: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<47, 3>);
    case 48: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<48, 3>);
    case 49: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<49, 3>);
    case 50: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<50, 3>);
    case 51: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<51, 3>);
    case 52: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<52, 3>);
    case 53: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<53, 3>);
    case 54: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<54, 3>);
    case 55: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<55, 3>);
    case 56: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<56, 3>);
    case 57: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<57, 3>);
    case 58: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<58, 3>);
    case 59: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<59, 3>);
    case 60: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<60, 3>);
    case 61: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<61, 3>);
    case 62: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<62, 3>);
    case 63: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<63, 3>);
    case 64: return reinterpret_cast<const void*>(&ryser_dense_tc_kernel<64, 3>);
    default: return nullptr;
  }
}
}  // namespace perm
