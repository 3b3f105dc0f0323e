// Host-only check of the tcgen05 descriptors the tensor-core matvecs build by
// hand (matvec_tc.cuh: idesc_tf32, desc_sw128; matvec_oz.cuh: idesc_i8),
// against CUTLASS's own sm100 descriptor constructors (cute/arch/
// mma_sm100_desc.hpp, from a CUTLASS include tree given with -I):
//   * the instruction descriptor of kind::i8 (signed INT8 x signed INT8 ->
//     S32) and of kind::tf32 (TF32 x TF32 -> F32), A and B K-major, M = 128,
//     for every N the kernels issue (16 ... 256 in steps of 16);
//   * the shared-memory descriptor of a K-major 128-byte-swizzled tile (start
//     address, LBO 16 B, SBO 1024 B, sm100 version 1, base offset 0) over
//     every 16-byte-aligned address of a 227 KB window.
// No CUDA call is made.  Usage: oz_desc_check (exit 0: all equal)
#include <cstdio>
#include <utility>

#include <cute/arch/mma_sm100_desc.hpp>

#include "matvec_oz.cuh"

static int fails = 0;

template <int N>
static void check_n()
{
  namespace U = cute::UMMA;
  const uint32_t i8 = uint32_t(U::make_instr_desc<int8_t, int8_t, int32_t, 128, N, U::Major::K, U::Major::K>());
  const uint32_t tf = uint32_t(U::make_instr_desc<cute::tfloat32_t, cute::tfloat32_t, float, 128, N, U::Major::K,
                                                  U::Major::K>());
  if (i8 != mbc::oz::idesc_i8(N)) {
    std::fprintf(stderr, "kind::i8 N=%d: cutlass %08x, ours %08x\n", N, i8, mbc::oz::idesc_i8(N));
    ++fails;
  }
  if (tf != mbc::tc::idesc_tf32(N)) {
    std::fprintf(stderr, "kind::tf32 N=%d: cutlass %08x, ours %08x\n", N, tf, mbc::tc::idesc_tf32(N));
    ++fails;
  }
}

template <int... I>
static void check_all(std::integer_sequence<int, I...>)
{
  (check_n<16 * (I + 1)>(), ...);
}

int main()
{
  check_all(std::make_integer_sequence<int, 16>{});  // N = 16 ... 256
  for (uint32_t a = 0; a < 232448u; a += 16) {
    cute::UMMA::SmemDescriptor d;
    d.start_address_ = (uint16_t)(a >> 4);
    d.leading_byte_offset_ = 1;
    d.stride_byte_offset_ = 1024 >> 4;
    d.version_ = 1;
    d.base_offset_ = 0;
    d.lbo_mode_ = 0;
    d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_128B);
    if (uint64_t(d) != mbc::tc::desc_sw128(a)) {
      if (fails < 10)
        std::fprintf(stderr, "smem descriptor at %u: cutlass %016llx, ours %016llx\n", a,
                     (unsigned long long)uint64_t(d), (unsigned long long)mbc::tc::desc_sw128(a));
      ++fails;
    }
  }
  if (fails) {
    std::fprintf(stderr, "%d descriptor mismatches\n", fails);
    return 1;
  }
  std::printf("all descriptors equal\n");
  return 0;
}
