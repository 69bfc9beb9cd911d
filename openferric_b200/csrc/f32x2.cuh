// Packed single-precision pairs: sm_100's add/sub/mul/fma .f32x2 instructions
// (PTX ISA 8.6) apply one IEEE round-to-nearest operation to both halves of a
// 64-bit register pair, so one issued instruction does the work of two.  Each
// half is rounded exactly as the scalar instruction would round it: code
// written with these gives the same bits as the scalar form with the same
// operation order (fma stays fma, a product followed by an add stays two
// roundings).
#pragma once

namespace of {

#define OF_F32X2_BINOP(NAME, OP)                                                               \
  __device__ __forceinline__ float2 NAME(float2 a, float2 b) {                                 \
    float2 d;                                                                                  \
    asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n " OP      \
        ".rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"                                      \
        : "=f"(d.x), "=f"(d.y)                                                                 \
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                             \
    return d;                                                                                  \
  }

OF_F32X2_BINOP(add2, "add")
OF_F32X2_BINOP(sub2, "sub")
OF_F32X2_BINOP(mul2, "mul")
#undef OF_F32X2_BINOP

// a * b + c with one rounding per half
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " mov.b64 rc, {%6, %7};\n fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}

__device__ __forceinline__ float2 splat2(float a) { return make_float2(a, a); }

}  // namespace of
