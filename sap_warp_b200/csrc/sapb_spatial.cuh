// sapb_spatial.cuh -- quaternion, transform and spatial-vector helpers (FP64)
// in the reference's conventions: quaternions xyzw, spatial vectors
// [angular; linear] at a body origin in world coordinates
// (sim/sap_helpers.py:576-1010).
#pragma once

#include <cuda_runtime.h>

namespace sapb {

struct V3 {
  double x, y, z;
};
struct Q4 {
  double x, y, z, w;
};
struct Xf {
  V3 p;
  Q4 q;
};
struct Sv {  // spatial vector [w; v]
  V3 w, v;
};

__device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 load3(const double* p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ void store3(double* p, V3 a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

__device__ __forceinline__ Q4 qident() { return Q4{0.0, 0.0, 0.0, 1.0}; }
__device__ __forceinline__ Q4 qmul(Q4 a, Q4 b) {
  return Q4{a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__device__ __forceinline__ Q4 qnormalize(Q4 q) {
  const double n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  if (!(n > 0.0)) return qident();
  const double r = 1.0 / n;
  return Q4{q.x * r, q.y * r, q.z * r, q.w * r};
}
__device__ __forceinline__ Q4 qconj(Q4 q) { return Q4{-q.x, -q.y, -q.z, q.w}; }
// rotate v by the unit quaternion q: v + w t + qv x t, t = 2 qv x v
__device__ __forceinline__ V3 qrot(Q4 q, V3 v) {
  const V3 qv = v3(q.x, q.y, q.z);
  const V3 t = 2.0 * cross(qv, v);
  return v + q.w * t + cross(qv, t);
}
__device__ __forceinline__ Q4 qaxis_angle(V3 axis, double angle) {
  const double h = 0.5 * angle;
  const double s = sin(h), c = cos(h);
  return Q4{axis.x * s, axis.y * s, axis.z * s, c};
}
__device__ __forceinline__ Xf xf_load(const double* p) { return Xf{v3(p[0], p[1], p[2]), Q4{p[3], p[4], p[5], p[6]}}; }
__device__ __forceinline__ Xf xf_compose(Xf a, Xf b) {
  const Q4 aq = qnormalize(a.q), bq = qnormalize(b.q);
  return Xf{a.p + qrot(aq, b.p), qnormalize(qmul(aq, bq))};
}
__device__ __forceinline__ Xf xf_inverse(Xf x) {
  const Q4 qi = qconj(qnormalize(x.q));
  return Xf{-qrot(qi, x.p), qi};
}

__device__ __forceinline__ Sv sv(V3 w, V3 v) { return Sv{w, v}; }
__device__ __forceinline__ Sv sv_zero() { return Sv{v3(0, 0, 0), v3(0, 0, 0)}; }
__device__ __forceinline__ Sv operator+(Sv a, Sv b) { return Sv{a.w + b.w, a.v + b.v}; }
__device__ __forceinline__ Sv operator*(double s, Sv a) { return Sv{s * a.w, s * a.v}; }
__device__ __forceinline__ double sdot(Sv a, Sv b) { return dot(a.w, b.w) + dot(a.v, b.v); }
__device__ __forceinline__ Sv sv_load(const double* p) { return Sv{v3(p[0], p[1], p[2]), v3(p[3], p[4], p[5])}; }
__device__ __forceinline__ void sv_store(double* p, Sv a) {
  store3(p, a.w);
  store3(p + 3, a.v);
}
// sim/sap_helpers.py:917-933
__device__ __forceinline__ Sv shift_velocity(Sv V, V3 p) { return Sv{V.w, V.v + cross(V.w, p)}; }
__device__ __forceinline__ Sv shift_acceleration(Sv A, V3 p, V3 w) {
  return Sv{A.w, A.v + cross(A.w, p) + cross(w, cross(w, p))};
}
__device__ __forceinline__ Sv shift_force(Sv F, V3 p) { return Sv{F.w - cross(p, F.v), F.v}; }
// sim/sap_helpers.py:936-994
__device__ __forceinline__ Sv compose_velocity(Sv V_WP, V3 p_PB, Sv V_PB) {
  return Sv{V_WP.w + V_PB.w, V_WP.v + cross(V_WP.w, p_PB) + V_PB.v};
}
__device__ __forceinline__ Sv compose_acceleration(Sv A_WP, Sv V_WP, V3 p_PB, Sv V_PB, Sv A_PB) {
  const V3 w = V_WP.w;
  const Sv As = shift_acceleration(A_WP, p_PB, w);
  return Sv{As.w + A_PB.w + cross(w, V_PB.w), As.v + A_PB.v + 2.0 * cross(w, V_PB.v)};
}
// sim/sap_helpers.py:997-1024
__device__ __forceinline__ Sv mobilizer_velocity_to_body(Q4 R_WF, V3 p_MoBo_F, Sv V_FM_F) {
  return Sv{qrot(R_WF, V_FM_F.w), qrot(R_WF, V_FM_F.v + cross(V_FM_F.w, p_MoBo_F))};
}
__device__ __forceinline__ Sv mobilizer_accel_bias_to_body(Q4 R_WF, V3 p_MoBo_F, V3 w_FM_F) {
  return Sv{v3(0, 0, 0), qrot(R_WF, cross(w_FM_F, cross(w_FM_F, p_MoBo_F)))};
}

// Rotation with the given columns (the reference's _quatd_from_matrix_cols,
// sim/sap_helpers.py:608-655: the trace branch, else the largest diagonal).
__device__ inline Q4 quat_from_cols(V3 c0, V3 c1, V3 c2) {
  const double r00 = c0.x, r10 = c0.y, r20 = c0.z, r01 = c1.x, r11 = c1.y, r21 = c1.z, r02 = c2.x, r12 = c2.y,
               r22 = c2.z;
  const double tr = r00 + r11 + r22;
  if (tr > 0.0) {
    const double s = sqrt(tr + 1.0) * 2.0;
    return Q4{(r21 - r12) / s, (r02 - r20) / s, (r10 - r01) / s, 0.25 * s};
  }
  if (r00 > r11 && r00 > r22) {
    const double s = sqrt(1.0 + r00 - r11 - r22) * 2.0;
    return Q4{0.25 * s, (r01 + r10) / s, (r02 + r20) / s, (r21 - r12) / s};
  }
  if (r11 > r22) {
    const double s = sqrt(1.0 + r11 - r00 - r22) * 2.0;
    return Q4{(r01 + r10) / s, 0.25 * s, (r12 + r21) / s, (r02 - r20) / s};
  }
  const double s = sqrt(1.0 + r22 - r00 - r11) * 2.0;
  return Q4{(r02 + r20) / s, (r12 + r21) / s, 0.25 * s, (r10 - r01) / s};
}

// D6 mobilizer (sim/sap_helpers.py:1109-1161, 1204-1241, 1247-1286,
// 1387-1431): `lin` translation axes a_k (coordinates q[0..lin)), then `ang`
// rotation axes; with two or three rotation axes each axis is carried by the
// rotations before it (axes e_x, e_y, e_z of the frame whose columns are the
// joint axes).  Writes the transform X_FM and the angular DOF axes in F.
__device__ inline void d6_mobilizer(const double* axes, const double* q, int lin, int ang, Xf* X, V3 ang_axis[3]) {
  V3 pos = v3(0, 0, 0);
  for (int k = 0; k < lin && k < 3; ++k) pos = pos + q[k] * load3(axes + 3 * k);
  Q4 rot = qident();
  const double* aa = axes + 3 * lin;
  const double* qa = q + lin;
  if (ang == 1) {
    ang_axis[0] = load3(aa);
    rot = qaxis_angle(ang_axis[0], qa[0]);
  } else if (ang == 2 || ang == 3) {
    const V3 c0 = load3(aa), c1 = load3(aa + 3);
    const V3 c2 = ang == 3 ? load3(aa + 6) : cross(c0, c1);
    const Q4 off = quat_from_cols(c0, c1, c2);
    const V3 l0 = qrot(off, v3(1, 0, 0)), l1 = qrot(off, v3(0, 1, 0)), l2 = qrot(off, v3(0, 0, 1));
    const Q4 q0 = qaxis_angle(l0, qa[0]);
    const V3 a1 = qrot(q0, l1);
    const Q4 q1 = qaxis_angle(a1, qa[1]);
    const Q4 q10 = qmul(q1, q0);
    ang_axis[0] = l0;
    ang_axis[1] = a1;
    rot = q10;
    if (ang == 3) {
      const V3 a2 = qrot(q10, l2);
      ang_axis[2] = a2;
      rot = qmul(qaxis_angle(a2, qa[2]), q10);
    }
  }
  X->p = pos;
  X->q = rot;
}

}  // namespace sapb
