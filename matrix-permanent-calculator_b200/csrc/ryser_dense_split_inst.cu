// ryser_dense_split_inst.cu -- instantiations of the split-X dense Ryser kernel,
// orders 4..40.
#include "ryser_dense_split.cuh"

namespace perm {
const void* dense_split_kernel(int n) {
  switch (n) {
    case 4: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<4>);
    case 5: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<5>);
    case 6: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<6>);
    case 7: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<7>);
    case 8: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<8>);
    case 9: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<9>);
    case 10: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<10>);
    case 11: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<11>);
    case 12: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<12>);
    case 13: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<13>);
    case 14: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<14>);
    case 15: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<15>);
    case 16: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<16>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<17>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<18>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<19>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<20>);
    case 21: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<21>);
    case 22: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<22>);
    case 23: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<23>);
    case 24: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<24>);
    case 25: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<25>);
    case 26: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<26>);
    case 27: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<27>);
    case 28: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<28>);
    case 29: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<29>);
    case 30: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<30>);
    case 31: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<31>);
    case 32: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<32>);
    case 33: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<33>);
    case 34: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<34>);
    case 35: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<35>);
    case 36: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<36>);
    case 37: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<37>);
    case 38: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<38>);
    case 39: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<39>);
    case 40: return reinterpret_cast<const void*>(&ryser_dense_split_kernel<40>);
    default: return nullptr;
  }
}
}  // namespace perm
