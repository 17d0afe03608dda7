// sapb_prepare.cu -- free motion and contact Jacobian of every world.
//
// Two launches per step:
//   scatter_contacts_kernel: each flat contact claims a slot in its world
//     (atomic, like _scatter_sap_contacts_to_env_direct,
//     sim/contact_jacobian.py:404-562); the world's CTA then re-ranks its
//     slots by flat contact index, so slot order is deterministic;
//   prepare_world_kernel: one CTA per world runs forward kinematics with
//     velocities and bias accelerations, body dynamics, the reverse force
//     pass, body Jacobians, A = sum_b J_b^T I_b J_b + armature, the free-motion
//     solve v* = v0 + dt A^-1 tau, and the contact slots' frames, phi0,
//     materials, Jacobian rows and weights -- everything the contact solve
//     reads (sim/free_motion.py:1804-2178, sim/contact_jacobian.py:1649-1985).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "sapb_internal.h"
#include "sapb_spatial.cuh"

namespace sapb {

constexpr int kPrepNT = 128;

struct PrepParams {
  sapb_model_desc m;
  sapb_step_inputs in;
  sapb_prepare_options o;
  sapb_prepare_outputs out;
  int32_t* env_count;  // [W]
  int32_t* env_src;    // [W][C]
  int32_t* truncated;  // [1]
};

__host__ __device__ inline size_t prep_align(size_t x) { return (x + 15) / 16 * 16; }

struct PrepLayout {
  size_t body, S, Jb, H, K, con, conint, bj, total;
};

__host__ __device__ inline PrepLayout prep_layout(int B, int n, int C) {
  PrepLayout L;
  size_t o = 0;
  L.body = o;  // pos3 quat4 V6 Ab6 fb6 ft6 I6[36] = 67 per body
  o = prep_align(o + sizeof(double) * 67 * (size_t)B);
  L.S = o;  // S[n][6], tau[n], vdot[n]
  o = prep_align(o + sizeof(double) * 8 * (size_t)n);
  L.Jb = o;
  o = prep_align(o + sizeof(double) * 6 * (size_t)B * n);
  L.H = o;
  o = prep_align(o + sizeof(double) * (size_t)n * n);
  L.K = o;
  o = prep_align(o + sizeof(double) * 6 * (size_t)n);
  L.con = o;  // per contact: xj0 3, xj1 3, p0 3, p1 3, F 9 = 21
  o = prep_align(o + sizeof(double) * 21 * (size_t)(C > 0 ? C : 1));
  L.conint = o;  // lb0, lb1
  o = prep_align(o + sizeof(int) * 2 * (size_t)(C > 0 ? C : 1));
  L.bj = o;  // body -> global joint
  o = prep_align(o + sizeof(int) * (size_t)B);
  L.total = o;
  return L;
}

__global__ void scatter_contacts_kernel(const PrepParams P) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int cap = P.in.contact_capacity;
  if (t >= cap) return;
  int live = P.in.contact_count[0];
  if (live > cap) live = cap;
  if (t >= live) return;
  const int sh0 = P.in.contact_shape0[t], sh1 = P.in.contact_shape1[t];
  const int S = P.m.num_shapes;
  const int b0 = (sh0 >= 0 && sh0 < S) ? P.m.shape_body[sh0] : -1;
  const int b1 = (sh1 >= 0 && sh1 < S) ? P.m.shape_body[sh1] : -1;
  const int B = P.m.bodies_per_world;
  const int nb = B * P.m.num_worlds;
  // _contact_env_from_shapes (sim/sap_helpers.py:439-464)
  int env = -1;
  if (b0 >= 0 && b0 < nb) env = b0 / B;
  else if (b1 >= 0 && b1 < nb) env = b1 / B;
  if (env < 0) return;
  if (b0 >= 0 && (b0 >= nb || b0 / B != env)) return;
  if (b1 >= 0 && (b1 >= nb || b1 / B != env)) return;
  const int slot = atomicAdd(&P.env_count[env], 1);
  if (slot < P.o.max_contacts)
    P.env_src[(size_t)env * P.o.max_contacts + slot] = t;
  else
    atomicAdd(P.truncated, 1);
}

// rows t1, t2, n of _sap_make_from_one_unit_vector_z (sim/sap_helpers.py:467-503)
__device__ inline void contact_frame(V3 n, double F[9]) {
  const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
  int i = 0;
  double mn = ax;
  if (ay < mn) {
    i = 1;
    mn = ay;
  }
  if (az < mn) {
    i = 2;
    mn = az;
  }
  const double mag = sqrt(1.0 - mn * mn);
  const double r = 1.0 / mag;
  const double umin = i == 0 ? n.x : (i == 1 ? n.y : n.z);
  const double s = -r * umin;
  V3 v, w;
  if (i == 0) {
    v = v3(0.0, -r * n.z, r * n.y);
    w = v3(mag, s * n.y, s * n.z);
  } else if (i == 1) {
    v = v3(r * n.z, 0.0, -r * n.x);
    w = v3(s * n.x, mag, s * n.z);
  } else {
    v = v3(-r * n.y, r * n.x, 0.0);
    w = v3(s * n.x, s * n.y, mag);
  }
  store3(F, v);
  store3(F + 3, w);
  store3(F + 6, n);
}

// material fallbacks (sim/sap_helpers.py:150-237)
__device__ inline double shape_mu(const PrepParams& P, int sh) {
  double v = P.o.fallback_mu;
  if (sh >= 0 && P.m.shape_material_mu) v = P.m.shape_material_mu[sh];
  return v < 0.0 ? 0.0 : v;
}
__device__ inline double shape_k(const PrepParams& P, int sh) {
  double v = P.o.fallback_stiffness;
  if (sh >= 0 && P.m.shape_material_ke) v = P.m.shape_material_ke[sh];
  if (!isfinite(v) || v <= 0.0) v = P.o.fallback_stiffness;
  if (!isfinite(v) || v <= 0.0) v = 1.0;
  return v;
}
__device__ inline double shape_tau(const PrepParams& P, int sh) {
  double v = P.o.fallback_tau_d;
  if (sh >= 0 && P.m.shape_material_tau) v = P.m.shape_material_tau[sh];
  if (!isfinite(v) || v < 0.0) v = P.o.fallback_tau_d;
  if (!isfinite(v) || v < 0.0) v = 0.0;
  return v;
}

__global__ void __launch_bounds__(kPrepNT) prepare_world_kernel(const PrepParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const int e = blockIdx.x;
  const int B = P.m.bodies_per_world, n = P.m.dofs_per_world, C = P.o.max_contacts;
  const int Jw = P.m.joints_per_world, Aw = P.m.articulations_per_world;
  const PrepLayout L = prep_layout(B, n, C);
  double* body = reinterpret_cast<double*>(smem + L.body);
  double* S = reinterpret_cast<double*>(smem + L.S);
  double* tau = S + 6 * n;
  double* vdot = tau + n;
  double* Jb = reinterpret_cast<double*>(smem + L.Jb);
  double* H = reinterpret_cast<double*>(smem + L.H);
  double* K = reinterpret_cast<double*>(smem + L.K);
  double* con = reinterpret_cast<double*>(smem + L.con);
  int* conint = reinterpret_cast<int*>(smem + L.conint);
  int* bj = reinterpret_cast<int*>(smem + L.bj);
  auto POS = [&](int b) { return body + 67 * b; };
  auto QUAT = [&](int b) { return body + 67 * b + 3; };
  auto VEL = [&](int b) { return body + 67 * b + 7; };
  auto ACC = [&](int b) { return body + 67 * b + 13; };
  auto FB = [&](int b) { return body + 67 * b + 19; };
  auto FT = [&](int b) { return body + 67 * b + 25; };
  auto I6 = [&](int b) { return body + 67 * b + 31; };
  const int j0 = e * Jw, b0g = e * B, d0 = e * n;

  for (int k = tid; k < 6 * n; k += kPrepNT) S[k] = 0.0;
  for (int k = tid; k < 6 * B * n; k += kPrepNT) Jb[k] = 0.0;
  for (int jl = tid; jl < Jw; jl += kPrepNT) {
    const int cb = P.m.joint_child[j0 + jl] - b0g;
    if (cb >= 0 && cb < B) bj[cb] = j0 + jl;
  }
  __syncthreads();

  // ---- forward kinematics, velocities, bias accelerations -----------------
  // One thread per articulation; joints in index order (parents first).
  // sim/free_motion.py:412-530 with sim/sap_helpers.py:1164-1433.
  for (int a = tid; a < Aw; a += kPrepNT) {
    const int ja = P.m.articulation_start[e * Aw + a], jb = P.m.articulation_start[e * Aw + a + 1];
    for (int j = ja; j < jb; ++j) {
      const int jt = P.m.joint_type[j];
      const int pb = P.m.joint_parent[j] >= 0 ? P.m.joint_parent[j] - b0g : -1;
      const int cb = P.m.joint_child[j] - b0g;
      const int qs = P.m.joint_q_start[j], ds = P.m.joint_qd_start[j], dl = ds - d0;
      const double* q = P.in.joint_q;
      const double* qd = P.in.joint_qd;
      const Xf Xp = xf_load(P.m.joint_X_p + 7 * (size_t)j);
      const Xf Xc = xf_load(P.m.joint_X_c + 7 * (size_t)j);
      Xf X_WF = Xp;
      if (pb >= 0) X_WF = xf_compose(Xf{load3(POS(pb)), Q4{QUAT(pb)[0], QUAT(pb)[1], QUAT(pb)[2], QUAT(pb)[3]}}, Xp);
      Xf X_FM{v3(0, 0, 0), qident()};
      Sv V_FM = sv_zero();
      if (jt == SAPB_JOINT_PRISMATIC) {
        const V3 ax = load3(P.m.joint_axis + 3 * (size_t)ds);
        X_FM.p = q[qs] * ax;
        V_FM = sv(v3(0, 0, 0), qd[ds] * ax);
      } else if (jt == SAPB_JOINT_REVOLUTE) {
        const V3 ax = load3(P.m.joint_axis + 3 * (size_t)ds);
        X_FM.q = qaxis_angle(ax, q[qs]);
        V_FM = sv(qd[ds] * ax, v3(0, 0, 0));
      } else if (jt == SAPB_JOINT_BALL) {
        X_FM.q = Q4{q[qs], q[qs + 1], q[qs + 2], q[qs + 3]};
        V_FM = sv(v3(qd[ds], qd[ds + 1], qd[ds + 2]), v3(0, 0, 0));
      } else if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
        X_FM.p = v3(q[qs], q[qs + 1], q[qs + 2]);
        X_FM.q = Q4{q[qs + 3], q[qs + 4], q[qs + 5], q[qs + 6]};
        V_FM = sv(v3(qd[ds], qd[ds + 1], qd[ds + 2]), v3(qd[ds + 3], qd[ds + 4], qd[ds + 5]));
      }
      const Xf X_WM = xf_compose(X_WF, X_FM);
      const Xf X_MB = xf_inverse(Xc);
      const Xf X_WB = xf_compose(X_WM, X_MB);
      const V3 p_MoBo_F = qrot(qnormalize(X_FM.q), X_MB.p);
      const Q4 R_WF = qnormalize(X_WF.q);
      // motion subspace columns
      if (jt == SAPB_JOINT_PRISMATIC) {
        sv_store(S + 6 * dl, mobilizer_velocity_to_body(R_WF, p_MoBo_F,
                                                        sv(v3(0, 0, 0), load3(P.m.joint_axis + 3 * (size_t)ds))));
      } else if (jt == SAPB_JOINT_REVOLUTE) {
        const V3 ax = load3(P.m.joint_axis + 3 * (size_t)ds);
        sv_store(S + 6 * dl, sv(qrot(R_WF, ax), qrot(R_WF, cross(ax, p_MoBo_F))));
      } else if (jt == SAPB_JOINT_BALL || jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
        const int cnt = jt == SAPB_JOINT_BALL ? 3 : 6;
        for (int k = 0; k < cnt; ++k) {
          double u[6] = {0, 0, 0, 0, 0, 0};
          u[k] = 1.0;
          sv_store(S + 6 * (dl + k), mobilizer_velocity_to_body(R_WF, p_MoBo_F, sv_load(u)));
        }
      }
      const Sv V_PB = mobilizer_velocity_to_body(R_WF, p_MoBo_F, V_FM);
      const Sv A_PB = mobilizer_accel_bias_to_body(R_WF, p_MoBo_F, V_FM.w);
      store3(POS(cb), X_WB.p);
      QUAT(cb)[0] = X_WB.q.x;
      QUAT(cb)[1] = X_WB.q.y;
      QUAT(cb)[2] = X_WB.q.z;
      QUAT(cb)[3] = X_WB.q.w;
      if (pb >= 0) {
        const Sv Vp = sv_load(VEL(pb)), Ap = sv_load(ACC(pb));
        const V3 p_PB = X_WB.p - load3(POS(pb));
        sv_store(VEL(cb), compose_velocity(Vp, p_PB, V_PB));
        sv_store(ACC(cb), compose_acceleration(Ap, Vp, p_PB, V_PB, A_PB));
      } else {
        sv_store(VEL(cb), V_PB);
        sv_store(ACC(cb), A_PB);
      }
    }
  }
  __syncthreads();

  // ---- body dynamics (sim/free_motion.py:680-719, sim/sap_helpers.py:1027-1105)
  for (int b = tid; b < B; b += kPrepNT) {
    const Q4 q = qnormalize(Q4{QUAT(b)[0], QUAT(b)[1], QUAT(b)[2], QUAT(b)[3]});
    const double m = P.m.body_mass[b0g + b];
    const double* Ic = P.m.body_inertia + 9 * (size_t)(b0g + b);
    const V3 c = qrot(q, load3(P.m.body_com + 3 * (size_t)(b0g + b)));
    // R Ic R^T with R's columns the rotated axes
    V3 col[3] = {qrot(q, v3(1, 0, 0)), qrot(q, v3(0, 1, 0)), qrot(q, v3(0, 0, 1))};
    double R[3][3], IW[3][3];
    for (int r = 0; r < 3; ++r) {
      R[r][0] = r == 0 ? col[0].x : (r == 1 ? col[0].y : col[0].z);
      R[r][1] = r == 0 ? col[1].x : (r == 1 ? col[1].y : col[1].z);
      R[r][2] = r == 0 ? col[2].x : (r == 1 ? col[2].y : col[2].z);
    }
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        double acc = 0.0;
        for (int u = 0; u < 3; ++u)
          for (int v = 0; v < 3; ++v) acc += R[r][u] * Ic[3 * u + v] * R[s][v];
        IW[r][s] = acc;
      }
    const double cc[3] = {c.x, c.y, c.z};
    const double cdc = dot(c, c);
    double* I = I6(b);
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        I[6 * r + s] = IW[r][s] + m * ((r == s ? cdc : 0.0) - cc[r] * cc[s]);
        I[6 * (r + 3) + (s + 3)] = r == s ? m : 0.0;
      }
    // m [c]x in the upper right, -m [c]x lower left
    const double cx[3][3] = {{0.0, -c.z, c.y}, {c.z, 0.0, -c.x}, {-c.y, c.x, 0.0}};
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        I[6 * r + (s + 3)] = m * cx[r][s];
        I[6 * (r + 3) + s] = -m * cx[r][s];
      }
    const Sv a = sv_load(ACC(b)), V = sv_load(VEL(b));
    double av[6], Ia[6];
    sv_store(av, a);
    for (int r = 0; r < 6; ++r) {
      double acc = 0.0;
      for (int s = 0; s < 6; ++s) acc += I[6 * r + s] * av[s];
      Ia[r] = acc;
    }
    const V3 w = V.w;
    const V3 Iw = v3(I[0] * w.x + I[1] * w.y + I[2] * w.z, I[6] * w.x + I[7] * w.y + I[8] * w.z,
                     I[12] * w.x + I[13] * w.y + I[14] * w.z);
    const V3 bias_t = cross(w, Iw);
    const V3 bias_f = m * cross(w, cross(w, c));
    const int world_g = e;
    const V3 g = load3(P.m.gravity + 3 * (size_t)world_g);
    const V3 fg = m * g;
    const V3 tg = cross(c, fg);
    double* fb = FB(b);
    fb[0] = Ia[0] + bias_t.x - tg.x;
    fb[1] = Ia[1] + bias_t.y - tg.y;
    fb[2] = Ia[2] + bias_t.z - tg.z;
    fb[3] = Ia[3] + bias_f.x - fg.x;
    fb[4] = Ia[4] + bias_f.y - fg.y;
    fb[5] = Ia[5] + bias_f.z - fg.z;
    for (int k = 0; k < 6; ++k) FT(b)[k] = 0.0;
  }
  __syncthreads();

  // ---- reverse pass (sim/free_motion.py:154-220, sim/sap_helpers.py:2090-2118)
  for (int a = tid; a < Aw; a += kPrepNT) {
    const int ja = P.m.articulation_start[e * Aw + a], jb = P.m.articulation_start[e * Aw + a + 1];
    for (int j = jb - 1; j >= ja; --j) {
      const int pb = P.m.joint_parent[j] >= 0 ? P.m.joint_parent[j] - b0g : -1;
      const int cb = P.m.joint_child[j] - b0g;
      const int ds = P.m.joint_qd_start[j], dl = ds - d0;
      const int dim = P.m.joint_dof_dim[2 * j] + P.m.joint_dof_dim[2 * j + 1];
      Sv f = sv_load(FB(cb)) + sv_load(FT(cb));
      if (P.in.body_f) f = f + sv_load(P.in.body_f + 6 * (size_t)(b0g + cb));
      for (int k = 0; k < dim; ++k) {
        const double jf = P.in.joint_f ? P.in.joint_f[ds + k] : 0.0;
        tau[dl + k] = -sdot(sv_load(S + 6 * (dl + k)), f) + jf;
      }
      if (pb >= 0) {
        const Sv sf = shift_force(f, load3(POS(pb)) - load3(POS(cb)));
        double* ft = FT(pb);
        ft[0] += sf.w.x;
        ft[1] += sf.w.y;
        ft[2] += sf.w.z;
        ft[3] += sf.v.x;
        ft[4] += sf.v.y;
        ft[5] += sf.v.z;
      }
    }
  }
  // ---- body Jacobians in world-local DOF numbering (sim/free_motion.py:722-765)
  for (int b = tid; b < B; b += kPrepNT) {
    int jj = bj[b];
    const V3 pb = load3(POS(b));
    while (jj >= 0) {
      const int colb = P.m.joint_child[jj] - b0g;
      const int dl = P.m.joint_qd_start[jj] - d0;
      const int dim = P.m.joint_dof_dim[2 * jj] + P.m.joint_dof_dim[2 * jj + 1];
      const V3 p = pb - load3(POS(colb));
      for (int k = 0; k < dim; ++k) {
        const Sv s = shift_velocity(sv_load(S + 6 * (dl + k)), p);
        double out[6];
        sv_store(out, s);
        for (int r = 0; r < 6; ++r) Jb[((size_t)b * 6 + r) * n + dl + k] = out[r];
      }
      jj = P.m.joint_ancestor[jj];
    }
  }
  for (int k = tid; k < n * n; k += kPrepNT) H[k] = 0.0;
  __syncthreads();

  // ---- A = sum_b J_b^T I_b J_b + armature (sim/free_motion.py:814-1179) ------
  for (int b = 0; b < B; ++b) {
    const double* I = I6(b);
    const double* Jbb = Jb + (size_t)b * 6 * n;
    for (int k = tid; k < 6 * n; k += kPrepNT) {
      const int r = k / n, col = k - r * n;
      double acc = 0.0;
      for (int s = 0; s < 6; ++s) acc += I[6 * r + s] * Jbb[(size_t)s * n + col];
      K[k] = acc;
    }
    __syncthreads();
    for (int k = tid; k < n * n; k += kPrepNT) {
      const int i = k / n, j = k - i * n;
      if (j > i) continue;
      double acc = 0.0;
      for (int r = 0; r < 6; ++r) acc += Jbb[(size_t)r * n + i] * K[(size_t)r * n + j];
      H[k] += acc;
    }
    __syncthreads();
  }
  double* Ag = P.out.dynamics_matrix + (size_t)e * n * n;
  for (int k = tid; k < n * n; k += kPrepNT) {
    const int i = k / n, j = k - i * n;
    double v = i >= j ? H[(size_t)i * n + j] : H[(size_t)j * n + i];
    if (i == j) v += P.m.joint_armature[d0 + i];
    Ag[k] = v;
  }
  __syncthreads();
  for (int i = tid; i < n; i += kPrepNT) H[(size_t)i * n + i] += P.m.joint_armature[d0 + i];
  __syncthreads();

  // ---- free-motion solve A vdot = tau (LDL^T, lower triangle) ---------------
  for (int k = 0; k < n; ++k) {
    const double rinv = 1.0 / H[(size_t)k * n + k];
    const int m = n - k - 1;
    const int cnt = m * (m + 1) / 2;
    for (int q = tid; q < cnt; q += kPrepNT) {
      int ii = (int)((sqrtf(8.0f * (float)q + 1.0f) - 1.0f) * 0.5f);
      while ((ii + 1) * (ii + 2) / 2 <= q) ++ii;
      while (ii * (ii + 1) / 2 > q) --ii;
      const int jj = q - ii * (ii + 1) / 2;
      const int i = k + 1 + ii, j = k + 1 + jj;
      H[(size_t)i * n + j] -= (H[(size_t)i * n + k] * rinv) * H[(size_t)j * n + k];
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int i = 0; i < n; ++i) {
      double s = tau[i];
      for (int k = 0; k < i; ++k) s -= (H[(size_t)i * n + k] / H[(size_t)k * n + k]) * vdot[k];
      vdot[i] = s;
    }
    for (int i = 0; i < n; ++i) vdot[i] /= H[(size_t)i * n + i];
    for (int i = n - 1; i >= 0; --i) {
      double s = vdot[i];
      for (int k = i + 1; k < n; ++k) s -= (H[(size_t)k * n + i] / H[(size_t)i * n + i]) * vdot[k];
      vdot[i] = s;
    }
  }
  __syncthreads();
  for (int i = tid; i < n; i += kPrepNT) {
    const double vd = vdot[i];
    P.out.v_star[d0 + i] = P.in.joint_qd[d0 + i] + P.in.dt[e] * vd;
    if (P.out.vdot) P.out.vdot[d0 + i] = vd;
  }
  if (P.out.body_q) {
    for (int b = tid; b < B; b += kPrepNT) {
      double* o = P.out.body_q + 7 * (size_t)(b0g + b);
      for (int k = 0; k < 3; ++k) o[k] = POS(b)[k];
      for (int k = 0; k < 4; ++k) o[3 + k] = QUAT(b)[k];
    }
  }

  // ---- contacts of this world ---------------------------------------------
  const int total = P.env_count[e];
  const int cc = total < C ? total : C;
  if (tid == 0 && P.out.contact_count) P.out.contact_count[e] = total;
  // Canonical slot order: the slots the scatter claimed in arrival order are
  // re-ranked by flat contact index (distinct), so an untruncated world's
  // slots follow the flat buffer's order on every step.
  {
    int* tmp = conint;  // 2*C ints, free until the rows below use them
    for (int c = tid; c < cc; c += kPrepNT) tmp[c] = P.env_src[(size_t)e * C + c];
    __syncthreads();
    for (int c = tid; c < cc; c += kPrepNT) {
      const int v = tmp[c];
      int rank = 0;
      for (int j = 0; j < cc; ++j) rank += tmp[j] < v ? 1 : 0;
      P.env_src[(size_t)e * C + rank] = v;
    }
    __syncthreads();
  }
  for (int c = tid; c < cc; c += kPrepNT) {
    const int src = P.env_src[(size_t)e * C + c];
    const int sh0 = P.in.contact_shape0[src], sh1 = P.in.contact_shape1[src];
    const int S_ = P.m.num_shapes;
    const int gb0 = (sh0 >= 0 && sh0 < S_) ? P.m.shape_body[sh0] : -1;
    const int gb1 = (sh1 >= 0 && sh1 < S_) ? P.m.shape_body[sh1] : -1;
    const int lb0 = gb0 >= 0 ? gb0 - b0g : -1, lb1 = gb1 >= 0 ? gb1 - b0g : -1;
    V3 x0 = load3(P.in.contact_point0 + 3 * (size_t)src);
    V3 x1 = load3(P.in.contact_point1 + 3 * (size_t)src);
    V3 p0 = v3(0, 0, 0), p1 = v3(0, 0, 0);
    if (lb0 >= 0) {
      p0 = load3(POS(lb0));
      x0 = p0 + qrot(qnormalize(Q4{QUAT(lb0)[0], QUAT(lb0)[1], QUAT(lb0)[2], QUAT(lb0)[3]}), x0);
    }
    if (lb1 >= 0) {
      p1 = load3(POS(lb1));
      x1 = p1 + qrot(qnormalize(Q4{QUAT(lb1)[0], QUAT(lb1)[1], QUAT(lb1)[2], QUAT(lb1)[3]}), x1);
    }
    V3 nrm = load3(P.in.contact_normal + 3 * (size_t)src);
    const double nn = sqrt(dot(nrm, nrm));
    if (nn > 0.0) nrm = (1.0 / nn) * nrm;
    double F[9];
    contact_frame(nrm, F);
    const double k0 = shape_k(P, sh0), k1 = shape_k(P, sh1);
    const double den = k0 + k1;
    double w0 = 0.5, w1 = 0.5;
    if (den != 0.0) {
      w0 = k0 / den;
      w1 = k1 / den;
    }
    const V3 pC = w0 * x0 + w1 * x1;
    const size_t ci = (size_t)e * C + c;
    const double m0 = P.in.contact_margin0 ? P.in.contact_margin0[src] : 0.0;
    const double m1 = P.in.contact_margin1 ? P.in.contact_margin1[src] : 0.0;
    P.out.phi0[ci] = dot(x1 - x0, nrm) - m0 - m1;
    const double mu0 = shape_mu(P, sh0), mu1 = shape_mu(P, sh1);
    const double mden = mu0 + mu1;
    P.out.mu[ci] = mden <= 1.0e-12 ? 0.0 : 2.0 * mu0 * mu1 / mden;
    double kc;
    if (!isfinite(k0)) kc = k1;
    else if (!isfinite(k1)) kc = k0;
    else kc = den <= 1.0e-12 ? fmax(k0, k1) : k0 * k1 / den;
    P.out.stiffness[ci] = kc;
    P.out.tau_d[ci] = shape_tau(P, sh0) + shape_tau(P, sh1);
    P.out.body0[ci] = gb0;
    P.out.body1[ci] = gb1;
    if (P.out.point) store3(P.out.point + 3 * ci, pC);
    if (P.out.frame)
      for (int k = 0; k < 9; ++k) P.out.frame[9 * ci + k] = F[k];
    double* cs = con + 21 * (size_t)c;
    const bool mid = P.o.contact_point_mode == SAPB_POINT_MIDPOINT;
    store3(cs + 0, mid ? pC : x0);
    store3(cs + 3, mid ? pC : x1);
    store3(cs + 6, p0);
    store3(cs + 9, p1);
    for (int k = 0; k < 9; ++k) cs[12 + k] = F[k];
    conint[2 * c] = lb0;
    conint[2 * c + 1] = lb1;
  }
  __syncthreads();
  double* Jout = P.out.jacobian + (size_t)e * C * 3 * n;
  for (int k = tid; k < cc * n; k += kPrepNT) {
    const int c = k / n, col = k - c * n;
    const double* cs = con + 21 * (size_t)c;
    V3 rel = v3(0, 0, 0);
    const int lb0 = conint[2 * c], lb1 = conint[2 * c + 1];
    if (lb1 >= 0) {
      const double* J = Jb + (size_t)lb1 * 6 * n + col;
      const V3 w = v3(J[0], J[n], J[2 * n]), v = v3(J[3 * n], J[4 * n], J[5 * n]);
      rel = rel + (v + cross(w, load3(cs + 3) - load3(cs + 9)));
    }
    if (lb0 >= 0) {
      const double* J = Jb + (size_t)lb0 * 6 * n + col;
      const V3 w = v3(J[0], J[n], J[2 * n]), v = v3(J[3 * n], J[4 * n], J[5 * n]);
      rel = rel - (v + cross(w, load3(cs + 0) - load3(cs + 6)));
    }
    for (int r = 0; r < 3; ++r) Jout[((size_t)c * 3 + r) * n + col] = dot(load3(cs + 12 + 3 * r), rel);
  }
  __syncthreads();
  // ---- contact weights (sim/contact_jacobian.py:153-251) --------------------
  for (int c = tid; c < cc; c += kPrepNT) {
    const size_t ci = (size_t)e * C + c;
    double w = 0.0;
    if (P.o.contact_weight_mode == SAPB_WEIGHT_DIAG_DELASSUS) {
      double w00 = 0, w01 = 0, w02 = 0, w11 = 0, w12 = 0, w22 = 0;
      const double* Jc = Jout + (size_t)c * 3 * n;
      for (int j = 0; j < n; ++j) {
        double aii = Ag[(size_t)j * n + j];
        if (aii < 1.0e-12) aii = 1.0e-12;
        const double inv = 1.0 / aii;
        const double a0 = Jc[j], a1 = Jc[n + j], a2 = Jc[2 * n + j];
        w00 += inv * a0 * a0;
        w01 += inv * a0 * a1;
        w02 += inv * a0 * a2;
        w11 += inv * a1 * a1;
        w12 += inv * a1 * a2;
        w22 += inv * a2 * a2;
      }
      w = sqrt(w00 * w00 + w11 * w11 + w22 * w22 + 2.0 * (w01 * w01 + w02 * w02 + w12 * w12)) / 3.0;
    } else {
      const double* cs = con + 21 * (size_t)c;
      const int lbs[2] = {conint[2 * c], conint[2 * c + 1]};
      // body-inertia weights use the witnesses, whatever the point mode
      const int src = P.env_src[ci];
      double wsum = 0.0;
      for (int side = 0; side < 2; ++side) {
        const int lb = lbs[side];
        if (lb < 0) continue;
        const double mass = P.m.body_mass[b0g + lb];
        if (mass <= 1.0e-12) continue;
        const Q4 q = qnormalize(Q4{QUAT(lb)[0], QUAT(lb)[1], QUAT(lb)[2], QUAT(lb)[3]});
        const V3 pb = load3(POS(lb));
        const V3 xw = pb + qrot(q, load3((side == 0 ? P.in.contact_point0 : P.in.contact_point1) + 3 * (size_t)src));
        const V3 com = pb + qrot(q, load3(P.m.body_com + 3 * (size_t)(b0g + lb)));
        const V3 r = xw - com;
        const double* Ic = P.m.body_inertia + 9 * (size_t)(b0g + lb);
        const double ix = fmax(Ic[0], 1.0e-12), iy = fmax(Ic[4], 1.0e-12), iz = fmax(Ic[8], 1.0e-12);
        for (int d = 0; d < 3; ++d) {
          const V3 cb = qrot(qconj(q), cross(r, load3(cs + 12 + 3 * d)));
          wsum += 1.0 / mass + cb.x * cb.x / ix + cb.y * cb.y / iy + cb.z * cb.z / iz;
        }
      }
      w = wsum / 3.0;
    }
    P.out.w_eff[ci] = w < 1.0e-12 ? 1.0e-12 : w;
  }
}

size_t prepare_smem_bytes(int B, int n, int C) { return prep_layout(B, n, C).total; }

int32_t prepare_launch(const sapb_model_desc* m, const sapb_step_inputs* in, const sapb_prepare_options* o,
                       const sapb_prepare_outputs* out, void* workspace, size_t workspace_bytes,
                       cudaStream_t stream) {
  PrepParams P;
  memset(&P, 0, sizeof(P));
  P.m = *m;
  P.in = *in;
  P.o = *o;
  P.out = *out;
  const int W = m->num_worlds, C = o->max_contacts;
  char* ws = static_cast<char*>(workspace);
  P.env_count = reinterpret_cast<int32_t*>(ws);
  P.truncated = P.env_count + W;
  P.env_src = P.truncated + 1;
  (void)workspace_bytes;
  if (W == 0) return SAPB_OK;
  cudaError_t err = cudaMemsetAsync(P.env_count, 0, sizeof(int32_t) * (W + 1), stream);
  if (err == cudaSuccess && in->contact_capacity > 0) {
    const int blocks = (in->contact_capacity + 255) / 256;
    scatter_contacts_kernel<<<blocks, 256, 0, stream>>>(P);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) {
    const size_t smem = prepare_smem_bytes(m->bodies_per_world, m->dofs_per_world, C);
    err = cudaFuncSetAttribute(prepare_world_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err == cudaSuccess) {
      prepare_world_kernel<<<W, kPrepNT, smem, stream>>>(P);
      err = cudaGetLastError();
    }
  }
  if (err == cudaSuccess && out->truncated_count)
    err = cudaMemcpyAsync(out->truncated_count, P.truncated, sizeof(int32_t), cudaMemcpyDeviceToDevice, stream);
  if (err != cudaSuccess) {
    set_last_error("free motion / contacts launch: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

// ---- position integration (sim/solver_sap.py:288-733) ----------------------
__global__ void integrate_kernel(const sapb_model_desc m, const double* q_in, const double* v_prev,
                                 const double* v_new, const double* dt, int mode, double* q_out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = m.joints_per_world * m.num_worlds;
  if (j >= J) return;
  const int jt = m.joint_type[j];
  const int qs = m.joint_q_start[j], ds = m.joint_qd_start[j];
  const int world = j / m.joints_per_world;
  const double h = dt[world];
  const bool mid = mode == SAPB_INTEGRATE_MIDPOINT;
  auto vel = [&](int k) { return mid ? 0.5 * (v_prev[k] + v_new[k]) : v_new[k]; };
  if (jt == SAPB_JOINT_PRISMATIC || jt == SAPB_JOINT_REVOLUTE) {
    q_out[qs] = q_in[qs] + h * vel(ds);
    return;
  }
  if (jt == SAPB_JOINT_FIXED) return;
  if (jt == SAPB_JOINT_BALL || jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
    const int o = jt == SAPB_JOINT_BALL ? 0 : 3;
    if (o == 3)
      for (int k = 0; k < 3; ++k) q_out[qs + k] = q_in[qs + k] + h * vel(ds + 3 + k);
    const Q4 q{q_in[qs + o], q_in[qs + o + 1], q_in[qs + o + 2], q_in[qs + o + 3]};
    const V3 w = v3(vel(ds), vel(ds + 1), vel(ds + 2));
    Q4 qn = q;
    if (!mid) {
      // qdot = 0.5 [0, w] q (sim/solver_sap.py:158-178)
      const double hd = 0.5 * h;
      qn = Q4{q.x + hd * (q.w * w.x + w.y * q.z - w.z * q.y), q.y + hd * (q.w * w.y + w.z * q.x - w.x * q.z),
              q.z + hd * (q.w * w.z + w.x * q.y - w.y * q.x), q.w - hd * (w.x * q.x + w.y * q.y + w.z * q.z)};
      const double nn = sqrt(qn.x * qn.x + qn.y * qn.y + qn.z * qn.z + qn.w * qn.w);
      if (nn > 0.0) qn = Q4{qn.x / nn, qn.y / nn, qn.z / nn, qn.w / nn};
    } else {
      // exp map of the midpoint angular velocity (sim/solver_sap.py:243-262)
      const double wn = sqrt(dot(w, w));
      const double angle = wn * h;
      if (angle > 1.0e-12) {
        const V3 axis = (1.0 / wn) * w;
        const Q4 r = qaxis_angle(axis, angle);
        qn = qmul(r, q);
        const double nn = sqrt(qn.x * qn.x + qn.y * qn.y + qn.z * qn.z + qn.w * qn.w);
        if (nn > 0.0) qn = Q4{qn.x / nn, qn.y / nn, qn.z / nn, qn.w / nn};
      }
    }
    q_out[qs + o] = qn.x;
    q_out[qs + o + 1] = qn.y;
    q_out[qs + o + 2] = qn.z;
    q_out[qs + o + 3] = qn.w;
    return;
  }
  // D6 and other multi-axis scalar joints: q += h * qd per axis
  const int dim = m.joint_dof_dim[2 * j] + m.joint_dof_dim[2 * j + 1];
  for (int k = 0; k < dim; ++k) q_out[qs + k] = q_in[qs + k] + h * vel(ds + k);
}

int32_t integrate_launch(const sapb_model_desc* m, const double* q_in, const double* v_prev, const double* v_new,
                         const double* dt, int mode, double* q_out, cudaStream_t stream) {
  const int J = m->joints_per_world * m->num_worlds;
  if (J == 0) return SAPB_OK;
  integrate_kernel<<<(J + 127) / 128, 128, 0, stream>>>(*m, q_in, v_prev, v_new, dt, mode, q_out);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error("integrate launch: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

}  // namespace sapb
