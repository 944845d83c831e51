// ryser_dense_inst_0.cu -- instantiations of the dense Ryser kernel for
// orders 1..20 (split across files so they compile in parallel).
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_0(int n) {
  switch (n) {
    case 1: return reinterpret_cast<const void*>(&ryser_dense_kernel<1>);
    case 2: return reinterpret_cast<const void*>(&ryser_dense_kernel<2>);
    case 3: return reinterpret_cast<const void*>(&ryser_dense_kernel<3>);
    case 4: return reinterpret_cast<const void*>(&ryser_dense_kernel<4>);
    case 5: return reinterpret_cast<const void*>(&ryser_dense_kernel<5>);
    case 6: return reinterpret_cast<const void*>(&ryser_dense_kernel<6>);
    case 7: return reinterpret_cast<const void*>(&ryser_dense_kernel<7>);
    case 8: return reinterpret_cast<const void*>(&ryser_dense_kernel<8>);
    case 9: return reinterpret_cast<const void*>(&ryser_dense_kernel<9>);
    case 10: return reinterpret_cast<const void*>(&ryser_dense_kernel<10>);
    case 11: return reinterpret_cast<const void*>(&ryser_dense_kernel<11>);
    case 12: return reinterpret_cast<const void*>(&ryser_dense_kernel<12>);
    case 13: return reinterpret_cast<const void*>(&ryser_dense_kernel<13>);
    case 14: return reinterpret_cast<const void*>(&ryser_dense_kernel<14>);
    case 15: return reinterpret_cast<const void*>(&ryser_dense_kernel<15>);
    case 16: return reinterpret_cast<const void*>(&ryser_dense_kernel<16>);
    case 17: return reinterpret_cast<const void*>(&ryser_dense_kernel<17>);
    case 18: return reinterpret_cast<const void*>(&ryser_dense_kernel<18>);
    case 19: return reinterpret_cast<const void*>(&ryser_dense_kernel<19>);
    case 20: return reinterpret_cast<const void*>(&ryser_dense_kernel<20>);
    default: return nullptr;
  }
}
}  // namespace perm
