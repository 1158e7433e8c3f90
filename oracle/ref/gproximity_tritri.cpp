// Thin host-side wrapper that compiles the reference's own gProximity tri-tri
// predicate (Source/Externals/inc/gProximity/cuda_intersect_tritri.h,
// triangleIntersection2 at :349-433) with g++ so the oracle's FP32 SAT
// restatement can be checked against it bit for bit.
// TEST INFRASTRUCTURE ONLY; the header is read from the reference tree at
// build time (oracle/ref/build.sh) and never copied into this repository.
#include <cfloat>
#include <cmath>
using std::fmax;
using std::fmin;
#include <vector_types.h>
#include <vector_functions.h>
#ifndef __device__
#define __device__
#endif
#ifndef __inline__
#define __inline__ inline
#endif
#include "cuda_intersect_tritri.h"

extern "C" int ref_tritri(const float *P, const float *Q) {
    return triangleIntersection2(make_float3(P[0], P[1], P[2]), make_float3(P[3], P[4], P[5]),
                                 make_float3(P[6], P[7], P[8]), make_float3(Q[0], Q[1], Q[2]),
                                 make_float3(Q[3], Q[4], Q[5]), make_float3(Q[6], Q[7], Q[8]));
}

extern "C" void ref_narrow(long long n, const int *pairs, const int *faces, const float *verts,
                           unsigned char *hit) {
    for (long long q = 0; q < n; q++) {
        float a[9], b[9];
        for (int k = 0; k < 3; k++)
            for (int c = 0; c < 3; c++) {
                a[3 * k + c] = verts[3 * (long long)faces[3 * (long long)pairs[2 * q] + k] + c];
                b[3 * k + c] = verts[3 * (long long)faces[3 * (long long)pairs[2 * q + 1] + k] + c];
            }
        hit[q] = (unsigned char)ref_tritri(a, b);
    }
}
