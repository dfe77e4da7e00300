// GPU check of the branch-free division used by the per-pixel loops
// (word2world_b200/csrc/common.cuh: rcp_markstein, div_markstein,
// div_in_range) against CUDA's correctly rounded __frcp_rn / __fdiv_rn.
//
//   * reciprocal: every significand, both signs, at several exponents;
//   * division: 2^32+ seeded random operand pairs per exponent range, counted
//     only where div_in_range admits them.
// Prints one line per case and exits 0 only when nothing differs.
#include <cstdint>
#include <cstdio>

#include "../../word2world_b200/csrc/common.cuh"

__global__ void rcp_check(int exp_shift, unsigned long long* bad, unsigned* first) {
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (1u << 23)) return;
  for (uint32_t sgn = 0; sgn < 2; ++sgn) {
    const uint32_t bits = (sgn << 31) | (uint32_t(127 + exp_shift) << 23) | m;
    const float b = __uint_as_float(bits);
    if (__float_as_uint(w2w::rcp_markstein(b)) != __float_as_uint(__frcp_rn(b))) {
      if (atomicAdd(bad, 1ull) == 0) *first = bits;
    }
  }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

__global__ void div_check(uint32_t seed, int iters, int ea_lo, int ea_hi, int eb_lo, int eb_hi,
                          unsigned long long* bad, unsigned long long* tested, uint2* last) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nb = 0, nt = 0;
  for (int i = 0; i < iters; ++i) {
    const uint32_t h1 = mix32(t * 2654435761u + uint32_t(i) * 40503u + seed);
    const uint32_t h2 = mix32(h1 ^ 0x9e3779b9u);
    const uint32_t h3 = mix32(h2 + 0x85ebca6bu);
    const int ea = ea_lo + int(h3 % uint32_t(ea_hi - ea_lo + 1));
    const int eb = eb_lo + int((h3 >> 16) % uint32_t(eb_hi - eb_lo + 1));
    const float a = __uint_as_float((h1 & 0x807fffffu) | (uint32_t(127 + ea) << 23));
    const float b = __uint_as_float((h2 & 0x807fffffu) | (uint32_t(127 + eb) << 23));
    if (!w2w::div_in_range(a, b)) continue;
    ++nt;
    if (__float_as_uint(w2w::div_markstein(a, b)) != __float_as_uint(__fdiv_rn(a, b))) {
      ++nb;
      *last = make_uint2(__float_as_uint(a), __float_as_uint(b));
    }
  }
  atomicAdd(bad, nb);
  atomicAdd(tested, nt);
}

int main(int argc, char** argv) {
  const int reps = argc > 1 ? atoi(argv[1]) : 4;
  unsigned long long *bad, *tested;
  unsigned* first;
  uint2* last;
  cudaMalloc(&bad, 8);
  cudaMalloc(&tested, 8);
  cudaMalloc(&first, 4);
  cudaMalloc(&last, 8);
  unsigned long long total_bad = 0;
  const int shifts[] = {-20, -7, -6, -5, -4, -3, -2, -1, 0, 1, 7, 20, 40, 60};
  for (int s : shifts) {
    cudaMemset(bad, 0, 8);
    cudaMemset(first, 0, 4);
    rcp_check<<<(1 << 23) / 256, 256>>>(s, bad, first);
    unsigned long long hb = 0;
    unsigned hf = 0;
    cudaMemcpy(&hb, bad, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&hf, first, 4, cudaMemcpyDeviceToHost);
    printf("reciprocal exponent %+d: mismatches %llu (first %08x)\n", s, hb, hf);
    total_bad += hb;
  }
  struct Range { int ea_lo, ea_hi, eb_lo, eb_hi; };
  const Range ranges[] = {{-60, 100, -20, 60}, {-10, 40, -4, 40}, {0, 30, -3, 12}, {-30, 0, -20, 0}};
  for (const Range& r : ranges) {
    cudaMemset(bad, 0, 8);
    cudaMemset(tested, 0, 8);
    for (int rep = 0; rep < reps; ++rep)
      div_check<<<148 * 64, 256>>>(1234u + 7919u * rep, 256, r.ea_lo, r.ea_hi, r.eb_lo, r.eb_hi, bad, tested, last);
    unsigned long long hb = 0, ht = 0;
    cudaMemcpy(&hb, bad, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&ht, tested, 8, cudaMemcpyDeviceToHost);
    printf("division a exp [%d,%d] b exp [%d,%d]: tested %llu mismatches %llu\n", r.ea_lo, r.ea_hi, r.eb_lo,
           r.eb_hi, ht, hb);
    total_bad += hb;
  }
  const cudaError_t e = cudaDeviceSynchronize();
  printf("status %s, total mismatches %llu\n", cudaGetErrorString(e), total_bad);
  return (e == cudaSuccess && total_bad == 0) ? 0 : 1;
}
