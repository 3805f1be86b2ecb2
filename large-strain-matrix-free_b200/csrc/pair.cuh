// Two FP32 values in one 64-bit register, operated on by the sm_100
// packed-FP32 instructions (add / sub / mul / fma .rn.f32x2): one issued
// instruction does the arithmetic of two cells.  The cell kernels are
// templates in their number type, so instantiating them with f2 runs the
// same sum factorisation and quadrature-point physics on a pair of cells
// (component x = first cell, y = second cell) at half the arithmetic issue
// slots.
//
// a * b yields a lazy product, so that `s += a * b` and `a * b + c * d`
// compile to fma.rn.f32x2 the way the compiler contracts scalar code.
#pragma once
#include <cstdint>
#include <cstring>

namespace lsmf {

struct f2 {
  unsigned long long v;
  f2() = default;
  __host__ __device__ f2(float a) { v = bcast_bits(a); }
  __host__ __device__ f2(double a) { v = bcast_bits((float)a); }
  __host__ __device__ f2(int a) { v = bcast_bits((float)a); }
  static __host__ __device__ unsigned long long bcast_bits(float a) {
#ifdef __CUDA_ARCH__
    unsigned long long r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
    return r;
#else
    uint32_t u;
    std::memcpy(&u, &a, 4);
    return ((unsigned long long)u << 32) | u;
#endif
  }
  static __device__ __forceinline__ f2 raw(unsigned long long bits) {
    f2 r;
    r.v = bits;
    return r;
  }
};

__device__ __forceinline__ f2 pack2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return f2::raw(r);
}
__device__ __forceinline__ void unpack2(f2 p, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(p.v));
}
__device__ __forceinline__ float lo2(f2 p) { float a, b; unpack2(p, a, b); return a; }
__device__ __forceinline__ float hi2(f2 p) { float a, b; unpack2(p, a, b); return b; }

__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
  return f2::raw(d);
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
  return f2::raw(d);
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.v), "l"(b.v));
  return f2::raw(d);
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a.v), "l"(b.v), "l"(c.v));
  return f2::raw(d);
}
// sign flip of both halves (there is no packed negation instruction)
__device__ __forceinline__ f2 neg2(f2 a) { return f2::raw(a.v ^ 0x8000000080000000ull); }

// lazy product a * b
struct f2p {
  f2 a, b;
  __device__ __forceinline__ operator f2() const { return mul2(a, b); }
};

__device__ __forceinline__ f2p operator*(f2 a, f2 b) { return {a, b}; }
__device__ __forceinline__ f2 operator+(f2 a, f2 b) { return add2(a, b); }
__device__ __forceinline__ f2 operator-(f2 a, f2 b) { return sub2(a, b); }
__device__ __forceinline__ f2 operator-(f2 a) { return neg2(a); }
__device__ __forceinline__ f2 operator+(f2p p, f2 c) { return fma2(p.a, p.b, c); }
__device__ __forceinline__ f2 operator+(f2 c, f2p p) { return fma2(p.a, p.b, c); }
__device__ __forceinline__ f2 operator+(f2p p, f2p q) { return fma2(q.a, q.b, mul2(p.a, p.b)); }
__device__ __forceinline__ f2 operator-(f2 c, f2p p) { return fma2(neg2(p.a), p.b, c); }
__device__ __forceinline__ f2 operator-(f2p p, f2 c) { return fma2(p.a, p.b, neg2(c)); }
__device__ __forceinline__ f2 operator-(f2p p, f2p q) { return fma2(neg2(q.a), q.b, mul2(p.a, p.b)); }
__device__ __forceinline__ f2p operator*(f2p p, f2 b) { return {mul2(p.a, p.b), b}; }
__device__ __forceinline__ f2p operator*(f2 a, f2p p) { return {a, mul2(p.a, p.b)}; }
__device__ __forceinline__ f2p operator*(f2p p, f2p q) { return {mul2(p.a, p.b), mul2(q.a, q.b)}; }
__device__ __forceinline__ f2 operator-(f2p p) { return mul2(neg2(p.a), p.b); }
__device__ __forceinline__ f2 operator/(f2 a, f2 b) {
  float a0, a1, b0, b1;
  unpack2(a, a0, a1);
  unpack2(b, b0, b1);
  return pack2(a0 / b0, a1 / b1);
}
__device__ __forceinline__ f2 operator/(f2p p, f2 b) { return f2(p) / b; }
__device__ __forceinline__ f2 &operator+=(f2 &c, f2p p) { return c = fma2(p.a, p.b, c); }
__device__ __forceinline__ f2 &operator+=(f2 &c, f2 a) { return c = add2(c, a); }
__device__ __forceinline__ f2 &operator-=(f2 &c, f2p p) { return c = fma2(neg2(p.a), p.b, c); }
__device__ __forceinline__ f2 &operator-=(f2 &c, f2 a) { return c = sub2(c, a); }
__device__ __forceinline__ f2 &operator*=(f2 &c, f2 a) { return c = mul2(c, a); }

// The records of two cells read as one: element i is the pair
// (first[i], second[i]).
struct RecPair {
  const float *p0, *p1;
  __device__ __forceinline__ f2 operator[](int i) const { return pack2(__ldg(p0 + i), __ldg(p1 + i)); }
  __device__ __forceinline__ RecPair operator+(int i) const { return {p0 + i, p1 + i}; }
};

}  // namespace lsmf
