// Test program: the kernels' division helpers against IEEE division, bit for
// bit, on the GPU. Prints one line per batch and exits 1 on any mismatch.
//   hfa::div_recip  (reciprocal + Markstein correction, fixed divisor)
//   hfa::div_rn     (zero-safe a / b)
//   hfa::div_rn_pos (a / b for b > 0)
// Inputs: counter-based random pairs; divisors from typical grid spacings,
// random ones within 2^+-100, and ones with exponents anywhere within 2^+-520
// (weighted towards 2^+-500); numerators over the whole exponent range with
// extra weight on the edges of div_recip's fast-path window and on
// 2^+-500, zeros, subnormals, infinities.
#include <cstdio>
#include <cuda_runtime.h>

#include "../../hydroflux_b200/csrc/hf_arith.h"

__device__ __forceinline__ unsigned long long mix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ bool same(double x, double y) {
  return __double_as_longlong(x) == __double_as_longlong(y) || (x != x && y != y);
}

__global__ void k_check(unsigned long long seed, long long n, int dmode,
                        unsigned long long* counts) {
  unsigned long long bad_recip = 0, bad_rn = 0, bad_pos = 0, fast = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r1 = mix(seed * 0x1000003ull + (unsigned long long)i);
    const unsigned long long r2 = mix(r1);
    double d;
    if (dmode == 0) {
      const double sp[8] = {1.0, 2.0, 5.0, 10.0, 30.0, 0.1, 3.7, 0.25};
      d = sp[r2 & 7];
    } else if (dmode == 1) {
      const unsigned long long e = 1023 - 100 + (r2 % 201);
      d = __longlong_as_double((long long)((e << 52) | ((r2 >> 11) & 0xFFFFFFFFFFFFFull)));
    } else {  // wide divisors, weighted towards 2^+-500
      const unsigned long long e = (r2 & 1) ? 1023 - 520 + (r2 % 1041)
                                            : ((r2 & 2) ? 523 - 8 : 1523 - 8) + (r2 >> 56) % 17;
      d = __longlong_as_double((long long)((e << 52) | ((r2 >> 11) & 0xFFFFFFFFFFFFFull)));
    }
    unsigned long long ea;
    const unsigned sel = (unsigned)(r1 >> 60);
    if (sel < 7) ea = 1023 - 60 + ((r1 >> 40) % 120);
    else if (sel < 9) ea = 1023 - 705 + ((r1 >> 40) % 12);
    else if (sel < 11) ea = 1023 + 895 + ((r1 >> 40) % 12);
    else if (sel < 13) ea = ((r1 >> 38) & 1 ? 523 - 8 : 1523 - 8) + ((r1 >> 40) % 17);
    else ea = (r1 >> 40) % 2048;  // anything: zeros, subnormals, inf / NaN
    const double a = __longlong_as_double(
        (long long)(((r1 & 1ull) << 63) | (ea << 52) | ((r1 >> 1) & 0xFFFFFFFFFFFFFull)));
    double num = a;
    asm volatile("" : "+d"(num));
    const double ref = num / d;
    const hfa::RecipD R = hfa::make_recip(d);
    const int e = hfa::biased_exponent(a);
    if (R.ok && e >= 1023 - 700 && e <= 1023 + 900) ++fast;
    if (!same(hfa::div_recip(a, R), ref)) ++bad_recip;
    if (!same(hfa::div_rn_pos(a, d), ref)) ++bad_pos;
    // div_rn with any divisor, zeros and specials included
    const double b = (r2 >> 63) ? -d : ((r2 & 0x30) == 0x30 ? 0.0 : d);
    double num2 = a;
    asm volatile("" : "+d"(num2));
    if (!same(hfa::div_rn(a, b), num2 / b)) ++bad_rn;
  }
  atomicAdd(&counts[0], bad_recip);
  atomicAdd(&counts[1], bad_pos);
  atomicAdd(&counts[2], bad_rn);
  atomicAdd(&counts[3], fast);
}

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : (1ll << 28);
  unsigned long long* counts = nullptr;
  if (cudaMalloc(&counts, 4 * sizeof(unsigned long long)) != cudaSuccess) return 2;
  int fails = 0;
  for (int dmode = 0; dmode < 3; ++dmode)
    for (unsigned long long seed = 1; seed <= 2; ++seed) {
      cudaMemset(counts, 0, 4 * sizeof(unsigned long long));
      k_check<<<148 * 8, 256>>>(seed + 10 * dmode, n, dmode, counts);
      unsigned long long h[4] = {0, 0, 0, 0};
      if (cudaMemcpy(h, counts, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
      printf("divisors %s, seed %llu: %lld pairs (%llu on the reciprocal fast path); "
             "mismatches div_recip %llu, div_rn_pos %llu, div_rn %llu\n",
             dmode == 0 ? "spacings" : (dmode == 1 ? "random" : "window"), seed, n, h[3], h[0],
             h[1], h[2]);
      fails += (h[0] || h[1] || h[2]);
    }
  return fails ? 1 : 0;
}
