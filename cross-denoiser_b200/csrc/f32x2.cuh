// Packed FP32x2 arithmetic on sm_100a (fma/mul/add/sub .rn.f32x2): one
// instruction for two lanes of fp32 data, each lane rounded as the scalar
// IEEE instruction, so packed code is bit-identical to scalar code with the
// same operation order.  The FMA pipe executes a pair in two cycles: the gain
// is issue bandwidth.  Used for the two buffers A and B of the spatial filter
// (filter_sweep.cuh) and of the block reconstruction (regression.cu), which
// share every tap or centre.
#pragma once
#include <cuda_runtime.h>
#include "cd_common.cuh"

namespace cd {
namespace x2 {

typedef unsigned long long f2;   // two floats: low half = buffer A, high half = buffer B

CD_DEV f2 pack(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
CD_DEV float lo(f2 v)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    (void)b;
    return a;
}
CD_DEV float hi(f2 v)
{
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    (void)a;
    return b;
}
CD_DEV f2 fma2(f2 a, f2 b, f2 c)
{
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
CD_DEV f2 mul2(f2 a, f2 b)
{
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
CD_DEV f2 add2(f2 a, f2 b)
{
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
CD_DEV f2 sub2(f2 a, f2 b)
{
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// |v|^2 of three pairs as the scalar norm2 rounds it: fma(z, z, fma(x, x, y*y))
CD_DEV f2 sqnorm2(f2 x, f2 y, f2 z) { return fma2(z, z, fma2(x, x, mul2(y, y))); }

}  // namespace x2
}  // namespace cd
