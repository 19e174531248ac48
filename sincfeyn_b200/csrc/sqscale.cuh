/* sqscale.cuh -- one value of the scaling test (driver/main.c:86-97), shared by the device kernel
 * (sqb_k_scale in sqkern.cuh) and host builds of the generated kernels.
 *
 * Value j = 3 d + q: direction d gives the exponents e_i in -E..E (base-(2E+1) digits of d over the
 * parameters other than the fixed one), q the step kappa (q+1)/3; x_i = x0_i xs[q][e_i + E] and
 * meas = prod_{i != fixed} x_i in double-double, g = |(double)(ptq(x, 0) meas)|; 0 for d = 0. */
#pragma once
#include "sqdd.cuh"
#include "sqb_internal.h"

template<class P>
SQDD_M double sqb_scale_value(const sqb_scale_t &a, long j){
    const int B = 2*a.E + 1;
    const long d = j/3; const int q = (int)(j - 3*d);
    int e[SQB_SCALE_MAXN], nz = 0; long r = d;
    for(int i = 0; i < a.n; i++){
        if(i == a.fixed){ e[i] = 0; continue; }
        e[i] = (int)(r % B) - a.E; r /= B; nz += e[i] != 0;
    }
    if(!nz) return 0;
    sqdd x[SQB_SCALE_MAXN], meas(1.0), ab;
    for(int i = 0; i < a.n; i++){
        x[i] = sqdd(a.x0[i])*sqdd(a.xs[q*B + e[i] + a.E]);
        if(i != a.fixed) meas = meas*x[i];
    }
    const sqdd v = P::pt(x, sqdd(0.0), &ab);
    return fabs((v*meas).value());
}
