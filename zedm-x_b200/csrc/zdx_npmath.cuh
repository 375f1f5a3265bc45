// zdx_npmath.cuh -- numpy's own arithmetic on 3- and 4-vectors, as polyline.py's calls round on this
// platform: np.dot of two 3-vectors is fma(a2, b2, fma(a1, b1, a0 b0)) (its BLAS's fused chain),
// np.linalg.norm of a 3- or 4-vector is the square root of that chain, np.linalg.norm(x, axis=1) of an
// (n, 3) array (tri_normals, polyline.py:99-109) is the square root of a plain sum of squares, and
// np.cross and the elementwise ufuncs are the plain IEEE operations.  fma is the IEEE fused
// multiply-add on the host and on the device alike.  The building block of a polyline mode bit-exact
// with polyline.py; host and device code, checked against numpy by tests/test_npmath_cpu.py.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define ZDX_HD_NP __host__ __device__ inline
#else
#define ZDX_HD_NP inline
#endif

namespace zdx {
namespace np {

// np.dot(a, b) of two 3-vectors
ZDX_HD_NP double dot3(const double* a, const double* b) { return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])); }

// np.linalg.norm(a) of a 3-vector
ZDX_HD_NP double norm3(const double* a) { return sqrt(dot3(a, a)); }

// np.linalg.norm(q) of a 4-vector (quat_normalize, polyline.py:36-41)
ZDX_HD_NP double norm4(const double* q) {
    return sqrt(fma(q[3], q[3], fma(q[2], q[2], fma(q[1], q[1], q[0] * q[0]))));
}

// one row of np.linalg.norm(x, axis=1) for an (n, 3) array
ZDX_HD_NP double row_norm3(const double* a) { return sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]); }

// np.cross(a, b) of two 3-vectors
ZDX_HD_NP void cross3(const double* a, const double* b, double* out) {
    const double x = a[1] * b[2] - a[2] * b[1];
    const double y = a[2] * b[0] - a[0] * b[2];
    const double z = a[0] * b[1] - a[1] * b[0];
    out[0] = x;
    out[1] = y;
    out[2] = z;
}

}  // namespace np
}  // namespace zdx
