// speedy_pk.cuh -- packed float32 pairs: sm_100's add/sub/mul on .f32x2 operands, two float32
// operations in one instruction.  Each lane is rounded to nearest on its own, exactly like the
// scalar instruction it replaces, so a packed expression gives the same bits as the two scalar
// expressions it pairs.  The lanes flush subnormal results to zero (.ftz), like the scalar
// arithmetic of the translation units that use them (speedy_ensemble.cu, the forward kernels,
// and speedy_selftest.cu, their check; both compiled with -ftz=true); code built without -ftz
// must not use these.
//
// One rule keeps the bits: ptxas contracts a packed add or subtract of a packed product into a
// fused multiply-add, whatever the rounding modifiers and -fmad say (measured on B200: the
// contracted sums differ from the separately rounded ones in about a quarter of random cases;
// an fma with a -0 addend or a unit factor in place of the multiply or the add is contracted the
// same way).  So pk_add / pk_sub take operands that are not products, and a sum with a product
// operand goes lane by lane through pk_add_sep / pk_sub_sep (two scalar operations, which are
// not contracted under -fmad=false).
//
// The forward is bound by instruction issue; the packed products and sums take one issue slot
// for two operations.
#pragma once

#include <cuda_runtime.h>

namespace spd {

#define SPD_PK_OP(name, op)                                                              \
  __device__ __forceinline__ float2 name(float2 a, float2 b) {                           \
    float2 d;                                                                            \
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t" \
        op " rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"                                  \
        : "=f"(d.x), "=f"(d.y)                                                           \
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                       \
    return d;                                                                            \
  }

SPD_PK_OP(pk_mul, "mul.rn.ftz.f32x2")
SPD_PK_OP(pk_add, "add.rn.ftz.f32x2")  // neither operand a product
SPD_PK_OP(pk_sub, "sub.rn.ftz.f32x2")  // neither operand a product
#undef SPD_PK_OP

// Sums with a product operand, lane by lane.
__device__ __forceinline__ float2 pk_add_sep(float2 a, float2 b) {
  return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 pk_sub_sep(float2 a, float2 b) {
  return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}

__device__ __forceinline__ float2 pk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 bc(float x) { return make_float2(x, x); }

}  // namespace spd
