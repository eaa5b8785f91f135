// pair_f32.cuh -- two single-precision lanes in one 64-bit register pair, computed with sm_100's packed FP32 instructions.
//
// The mixed-precision Jacobian action is issue-bound: every FP32 value of a point takes its own FFMA, its own shared-memory
// load and its own index arithmetic.  The paired kernel (k_ijacobian_pair) carries the same point of TWO elements of one
// colour in one f2: lane .x is the first element, lane .y the second, and every add / subtract / multiply / fused
// multiply-add is one packed instruction (add/sub/mul/fma .rn.f32x2) for both, with shared-memory values moved as 8-byte
// pairs.  Both lanes round exactly as the scalar FP32 code does (round-to-nearest per lane, products fused into adds where
// the scalar code fuses them); division and other non-packed operations run per lane.
//
// Fused multiply-adds: C++ operators cannot fuse a product into a later addition the way the compiler contracts a * b + c
// for scalars, so a * b returns a pending product (f2p) and the additive operators turn it into one packed FMA:
// a * b + c, c + a * b, a * b - c, c - a * b, s += a * b, s -= a * b.  Used anywhere else a pending product becomes a
// packed multiply.
#pragma once

#include <cuda_runtime.h>

namespace hb {

struct f2 {
  unsigned long long r;  // lanes packed as {x, y}
  f2() = default;
  __host__ __device__ f2(double d) { set(float(d), float(d)); }
  __host__ __device__ f2(float a, float b) { set(a, b); }
  __host__ __device__ void set(float a, float b) {
#ifdef __CUDA_ARCH__
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
#else
    unsigned ua, ub;
    __builtin_memcpy(&ua, &a, 4);
    __builtin_memcpy(&ub, &b, 4);
    r = (unsigned long long)ua | ((unsigned long long)ub << 32);
#endif
  }
  __device__ __forceinline__ float x() const { return __uint_as_float((unsigned)(r & 0xffffffffull)); }
  __device__ __forceinline__ float y() const { return __uint_as_float((unsigned)(r >> 32)); }
};

__device__ __forceinline__ f2 f2_raw(unsigned long long r) {
  f2 v;
  v.r = r;
  return v;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.r), "l"(b.r));
  return f2_raw(d);
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.r), "l"(b.r));
  return f2_raw(d);
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.r), "l"(b.r));
  return f2_raw(d);
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a.r), "l"(b.r), "l"(c.r));
  return f2_raw(d);
}
// 0 - a: one packed instruction (PTX has no packed negate); differs from -a only in the sign of a zero result
__device__ __forceinline__ f2 neg2(f2 a) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(0ull), "l"(a.r));
  return f2_raw(d);
}

// a pending product a * b
struct f2p {
  f2 a, b;
  __device__ __forceinline__ operator f2() const { return mul2(a, b); }
};

__device__ __forceinline__ f2p operator*(f2 a, f2 b) { return f2p{a, b}; }
__device__ __forceinline__ f2p operator*(f2p p, f2 c) { return f2p{mul2(p.a, p.b), c}; }
__device__ __forceinline__ f2p operator*(f2 c, f2p p) { return f2p{c, mul2(p.a, p.b)}; }
__device__ __forceinline__ f2p operator*(f2p p, f2p q) { return f2p{mul2(p.a, p.b), mul2(q.a, q.b)}; }

__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return add2(a, b); }
__device__ __forceinline__ f2 operator+(f2p p, f2 c) { return fma2(p.a, p.b, c); }
__device__ __forceinline__ f2 operator+(f2 c, f2p p) { return fma2(p.a, p.b, c); }
__device__ __forceinline__ f2 operator+(f2p p, f2p q) { return fma2(p.a, p.b, mul2(q.a, q.b)); }

__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return sub2(a, b); }
__device__ __forceinline__ f2 operator-(f2p p, f2 c) { return fma2(p.a, p.b, neg2(c)); }
__device__ __forceinline__ f2 operator-(f2 c, f2p p) { return fma2(neg2(p.a), p.b, c); }
__device__ __forceinline__ f2 operator-(f2p p, f2p q) { return fma2(p.a, p.b, neg2(mul2(q.a, q.b))); }

__device__ __forceinline__ f2 operator-(f2 a) { return neg2(a); }
__device__ __forceinline__ f2p operator-(f2p p) { return f2p{neg2(p.a), p.b}; }

__device__ __forceinline__ f2 &operator+=(f2 &s, f2 b) { return s = add2(s, b); }
__device__ __forceinline__ f2 &operator+=(f2 &s, f2p p) { return s = fma2(p.a, p.b, s); }
__device__ __forceinline__ f2 &operator-=(f2 &s, f2 b) { return s = sub2(s, b); }
__device__ __forceinline__ f2 &operator-=(f2 &s, f2p p) { return s = fma2(neg2(p.a), p.b, s); }
__device__ __forceinline__ f2 &operator*=(f2 &s, f2 b) { return s = mul2(s, b); }

// division per lane (IEEE single-precision quotient in each, as the scalar code computes it)
__device__ __forceinline__ f2 operator/(f2 a, f2 b) { return f2(a.x() / b.x(), a.y() / b.y()); }
__device__ __forceinline__ f2 operator/(f2p p, f2 b) { return f2(p) / b; }

}  // namespace hb
