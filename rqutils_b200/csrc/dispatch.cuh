// Compile-time dispatch over vector element types.
#pragma once
#include "common.cuh"

namespace sqd {

template <typename T>
struct TypeTag {
  using type = T;
};
template <int N>
struct IntTag {
  static constexpr int value = N;
};

// Calls f(TypeTag<R>, IntTag<NCV>, IntTag<NCA>): R = real type of the vector, NCV = 1/2 for a
// real/complex vector, NCA = 1/2 for real/complex matrix elements.
template <typename F>
void dispatch_vec(int dtype, int value_complex, F&& f) {
  switch (dtype) {
    case SQD_F64:
      SQD_REQUIRE(!value_complex, "a real vector dtype needs a Hamiltonian with real elements");
      f(TypeTag<double>{}, IntTag<1>{}, IntTag<1>{});
      break;
    case SQD_C128:
      if (value_complex) f(TypeTag<double>{}, IntTag<2>{}, IntTag<2>{});
      else f(TypeTag<double>{}, IntTag<2>{}, IntTag<1>{});
      break;
    case SQD_F32:
      SQD_REQUIRE(!value_complex, "a real vector dtype needs a Hamiltonian with real elements");
      f(TypeTag<float>{}, IntTag<1>{}, IntTag<1>{});
      break;
    case SQD_C64:
      if (value_complex) f(TypeTag<float>{}, IntTag<2>{}, IntTag<2>{});
      else f(TypeTag<float>{}, IntTag<2>{}, IntTag<1>{});
      break;
    default:
      throw Error(SQD_ERR_INVALID, "unknown dtype");
  }
}

template <typename F>
void dispatch_lpr(int lpr, F&& f) {
  switch (lpr) {
    case 1: f(IntTag<1>{}); break;
    case 2: f(IntTag<2>{}); break;
    case 4: f(IntTag<4>{}); break;
    case 8: f(IntTag<8>{}); break;
    case 16: f(IntTag<16>{}); break;
    case 32: f(IntTag<32>{}); break;
    default: throw Error(SQD_ERR_INVALID, "lanes per row must be 1, 2, 4, 8, 16 or 32");
  }
}

}  // namespace sqd
