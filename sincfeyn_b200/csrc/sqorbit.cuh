/* sqorbit.cuh -- the symmetry fold's per-point rules (driver/sum.c:29-46), shared by the device kernels
 * and host builds (the CPU tests compile this file as it is).
 *
 * A group element e maps k to its image k'_i = k[g[e][i]]; element 0 is the identity.  A point is
 * evaluated only if it is the lexicographic minimum of its orbit (symw()), and then weighs the orbit
 * size n / |stabiliser|; a kept point brings its whole orbit, the images in element order, each once
 * (symorbit()).  Axis indices are reduced modulo D, so no group can address outside k. */
#pragma once
#include "sqdd.cuh"
#include "sqb_internal.h"

/* symw() with D known at compile time: the image k[g[e][i]] is selected from the registers by an
 * unrolled compare, so k stays out of local memory in the register-bound evaluation kernels */
template<int D>
SQDD_M int sqb_orbit(const sqb_sym_t &s, const int (&k)[D]){
    int stab = 1;
    for(int e = 1; e < s.n; e++){
        int c = 0;
#pragma unroll
        for(int i = 0; i < D; i++){
            const int p = s.g[e][i];
            int y = k[0];
#pragma unroll
            for(int j = 1; j < D; j++) y = p == j ? k[j] : y;
            if(c == 0 && k[i] != y) c = k[i] < y ? -1 : 1;
        }
        if(c > 0) return 0;
        if(c == 0) stab++;
    }
    return s.n/stab;
}

/* symw() with D known at run time */
SQDD_M int sqb_orbit_n(const sqb_sym_t &s, const int *k, int D){
    int stab = 1;
    for(int e = 1; e < s.n; e++){
        int c = 0;
        for(int i = 0; i < D && !c; i++){ const int x = k[i], y = k[(unsigned)s.g[e][i] % (unsigned)D]; if(x != y) c = x < y ? -1 : 1; }
        if(c > 0) return 0;
        if(!c) stab++;
    }
    return s.n/stab;
}

/* the image of k under element e (e = 0: k itself) */
SQDD_M void sqb_image(const sqb_sym_t &s, const int *k, int D, int e, int *out){
    for(int d = 0; d < D; d++) out[d] = e ? k[(unsigned)s.g[e][d] % (unsigned)D] : k[d];
}

/* whether element e's image of k differs from the images of elements 0 .. e-1 (a new orbit member) */
SQDD_M bool sqb_image_new(const sqb_sym_t &s, const int *k, int D, int e){
    const unsigned uD = (unsigned)D;
    for(int f = 0; f < e; f++){
        bool eq = true;
        for(int d = 0; d < D && eq; d++) eq = k[(unsigned)s.g[e][d] % uD] == k[(unsigned)s.g[f][d] % uD];
        if(eq) return false;
    }
    return true;
}
