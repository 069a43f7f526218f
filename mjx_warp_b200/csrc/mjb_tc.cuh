// Warp-level tensor-core products in split TF32 ("3xTF32"): a float x is split into
// x = hi + lo with hi = tf32(x) (round to nearest, ties away) and lo = tf32(x - hi); a product
// a * b is then accumulated as a_lo * b_hi + a_hi * b_lo + a_hi * b_hi in FP32 by
// mma.sync.m16n8k8 (the a_lo * b_lo term, ~2^-22 relative, is dropped).  The result carries
// close to FP32 accuracy while the multiplies run on the tensor pipe.
//
// Fragment layout of mma.m16n8k8 with .tf32 operands (PTX ISA, "Matrix fragments for
// mma.m16n8k8"), g = lane / 4, t = lane % 4:
//   A (16 x 8, row major): a0 = A[g][t], a1 = A[g + 8][t], a2 = A[g][t + 4], a3 = A[g + 8][t + 4]
//   B (8 x 8, column major): b0 = B[t][g], b1 = B[t + 4][g]
//   C, D (16 x 8): c0 = C[g][2t], c1 = C[g][2t + 1], c2 = C[g + 8][2t], c3 = C[g + 8][2t + 1]
#pragma once

#include <cstdint>

namespace mjb {

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// x = hi + lo (+ the rounding error of lo), both TF32 values held in FP32 bit patterns
__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

// d += A * B for one m16n8k8 TF32 tile (FP32 accumulators)
__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// A fragment split into its hi and lo parts
struct FragA {
  uint32_t h[4], l[4];
};
struct FragB {
  uint32_t h[2], l[2];
};

__device__ __forceinline__ FragA frag_a(float a0, float a1, float a2, float a3) {
  FragA f;
  tf32_split(a0, f.h[0], f.l[0]);
  tf32_split(a1, f.h[1], f.l[1]);
  tf32_split(a2, f.h[2], f.l[2]);
  tf32_split(a3, f.h[3], f.l[3]);
  return f;
}
__device__ __forceinline__ FragB frag_b(float b0, float b1) {
  FragB f;
  tf32_split(b0, f.h[0], f.l[0]);
  tf32_split(b1, f.h[1], f.l[1]);
  return f;
}

// d += A * B in split TF32 (small terms first)
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const FragA& a, const FragB& b) {
  mma_tf32(d, a.l[0], a.l[1], a.l[2], a.l[3], b.h[0], b.h[1]);
  mma_tf32(d, a.h[0], a.h[1], a.h[2], a.h[3], b.l[0], b.l[1]);
  mma_tf32(d, a.h[0], a.h[1], a.h[2], a.h[3], b.h[0], b.h[1]);
}

}  // namespace mjb
