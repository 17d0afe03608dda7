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

#include "sapb_device.cuh"
#include "sapb_internal.h"
#include "sapb_joint.cuh"
#include "sapb_ldlt.cuh"
#include "sapb_spatial.cuh"

namespace sapb {

constexpr int kPrepNT = 128;
// per-contact scratch of the free-motion kernel: witness points x0, x1 (3
// each), then the contact frame (9)
constexpr int kConStride = 15;
constexpr int kConFrame = 6;

struct PrepParams {
  sapb_model_desc m;
  sapb_step_inputs in;
  sapb_prepare_options o;
  sapb_prepare_outputs out;
  int32_t* env_count;  // [W]
  int32_t* env_src;    // [W][C]
  int32_t* truncated;  // [1]
  // the contact history run before this kernel: slots already ranked, the
  // start impulses and known-impulse counts by slot (NULL: no history)
  bool ranked;
  const double* gamma_start;  // [W][C][3]
  const int32_t* hist_depth;  // [W][C]
};

__host__ __device__ inline size_t prep_align(size_t x) { return (x + 15) / 16 * 16; }

// Shared-memory layout of one world (doubles unless noted).  Spatial
// quantities are Plucker vectors about the world origin in world axes
// ([angular; linear]), so velocities, forces and inertias of different bodies
// add without shifts.
struct PrepLayout {
  size_t pose, pose2, fm, vj, cb, vb, fb, ib, fs, S, F, vec, H, con, conint, anc, jmp, bj, par, dbody, tri, jg,
      trees, total;
};

// tb: 0 for the dense layout, else the block size of the tree-blocked outputs
__host__ __device__ inline PrepLayout prep_layout(int B, int n, int C, int tb) {
  const bool blk = tb > 0;
  PrepLayout L;
  const size_t Cc = (size_t)(C > 0 ? C : 1);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = prep_align(o + bytes);
    return at;
  };
  L.pose = take(sizeof(double) * 8 * B);    // p 3, q 4 (pointer-jumping buffer A)
  L.pose2 = take(sizeof(double) * 8 * B);   // buffer B
  // The body arrays, dead once tau and the F columns are formed; A (tree
  // blocks when blocked) is formed after that and takes their bytes
  {
    const size_t body = (size_t)50 * B;  // vj 6, cb 6, vb 6, fb 6, ib 10, fs 16 per body
    const size_t h = blk ? (size_t)tb * tb * B : (size_t)n * n;
    const size_t at = take(sizeof(double) * (body > h ? body : h));
    L.vj = at;                                 // joint velocity S q_dot
    L.cb = at + sizeof(double) * 6 * B;        // joint bias acceleration
    L.vb = at + sizeof(double) * 12 * B;       // body velocity
    L.fb = at + sizeof(double) * 18 * B;       // body force
    L.ib = at + sizeof(double) * 24 * B;       // inertia: m, h = m c, I_O (xx yy zz xy xz yz)
    L.fs = at + sizeof(double) * 34 * B;       // subtree force 6 + composite inertia 10
    L.H = at;
  }
  L.S = take(sizeof(double) * 6 * n);       // motion subspace columns
  L.F = take(sizeof(double) * 6 * n);       // composite inertia times S
  L.vec = take(sizeof(double) * 4 * n);     // tau, vdot, diag(A), 1/d
  // per contact: x0 3, x1 3, frame 9; before the contacts are set up, X_FM
  // of each body's joint (8 per body) lives in the same bytes
  {
    const size_t con = (size_t)kConStride * Cc, fm = (size_t)8 * B;
    L.con = take(sizeof(double) * (con > fm ? con : fm));
    L.fm = L.con;
  }
  L.conint = take(sizeof(int) * 2 * Cc);    // local bodies lb0, lb1
  L.anc = take(sizeof(uint64_t) * 2 * B);   // ancestor-or-self masks (two buffers; then bodies by depth)
  L.jmp = take(sizeof(int) * 2 * B);        // pointer-jumping parents (two buffers)
  L.bj = take(sizeof(int) * B);             // joint (global index) of each body, -1
  L.par = take(sizeof(int) * B);            // parent body, -1
  L.dbody = take(sizeof(int) * n);          // body of each DOF
  L.tri = take(sizeof(uint16_t) * (blk ? 1 : (size_t)(n * (n - 1) / 2 + 1)));  // LDL^T triangle list
  L.jg = take(sizeof(double) * (blk ? 1 : (size_t)(kPrepNT / 32) * n));  // per-warp J^T gamma_start partials
  L.trees = take(sizeof(int) * (blk ? (size_t)2 * B + 1 : 1));  // tree of each body; first DOF of each tree
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
  // _contact_env_from_shapes (sim/sap_helpers.py:439-464)
  const int w0 = body_world_of(P.m, b0), w1 = body_world_of(P.m, b1);
  int env = -1;
  if (w0 >= 0) env = w0;
  else if (w1 >= 0) env = w1;
  if (env < 0) return;
  if (b0 >= 0 && w0 != env) return;
  if (b1 >= 0 && w1 != env) return;
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

// Spatial helpers about the world origin.
__device__ __forceinline__ Sv crm(Sv a, Sv b) {  // motion x motion
  return Sv{cross(a.w, b.w), cross(a.w, b.v) + cross(a.v, b.w)};
}
__device__ __forceinline__ Sv crf(Sv a, Sv f) {  // motion x* force
  return Sv{cross(a.w, f.w) + cross(a.v, f.v), cross(a.w, f.v)};
}
// Inertia (m, h = m c, I_O symmetric xx yy zz xy xz yz) times a motion vector.
__device__ __forceinline__ Sv inertia_times(const double* I, Sv m) {
  const V3 h = v3(I[1], I[2], I[3]);
  const V3 w = m.w;
  const V3 Iw = v3(I[4] * w.x + I[7] * w.y + I[8] * w.z, I[7] * w.x + I[5] * w.y + I[9] * w.z,
                   I[8] * w.x + I[9] * w.y + I[6] * w.z);
  return Sv{Iw + cross(h, m.v), I[0] * m.v - cross(h, w)};
}
__device__ __forceinline__ Xf pose_load(const double* p) {
  return Xf{v3(p[0], p[1], p[2]), Q4{p[3], p[4], p[5], p[6]}};
}
__device__ __forceinline__ void pose_store(double* p, Xf x) {
  p[0] = x.p.x;
  p[1] = x.p.y;
  p[2] = x.p.z;
  p[3] = x.q.x;
  p[4] = x.q.y;
  p[5] = x.q.z;
  p[6] = x.q.w;
}

// One CTA per world.  The tree recursions of the reference's free motion
// (sim/free_motion.py:412-1249, 1804-2178) become: poses by pointer jumping
// over the parent links (log depth rounds), per-joint motion subspaces and
// joint velocities in parallel, body velocities / bias accelerations as sums
// over ancestor masks, subtree forces and composite inertias by one pass
// from the deepest bodies up, A by the composite-rigid-body pairs H_ij = S_j . (I^c S_i),
// then a blocked LDL^T (diagonal blocks in registers) and block triangular solves.
// The contact rows are J_c = R_WC (v_O + w x x_c) of the ancestor DOFs' S
// columns (sim/contact_jacobian.py:404-562).
// VS: the candidate start velocity is written (v_start; a separate
// instantiation keeps its registers off the plain path).
template <bool VS>
__global__ void __launch_bounds__(kPrepNT, 7) prepare_world_kernel(const PrepParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const int e = blockIdx.x;
  const int C = P.o.max_contacts;
  const bool blk = P.o.tree_blocked != 0;  // tree-blocked outputs: the trees are the articulations
  const int tb = blk ? (P.o.tree_dofs > 0 ? P.o.tree_dofs : 6) : 0;  // their block size
  // shared memory laid out for the largest world; this world's own block
  const PrepLayout L = prep_layout(P.m.bodies_per_world, P.m.dofs_per_world, C, tb);
  const WorldSpan ws = world_span(P.m, e);
  const int B = ws.nb, n = ws.nd, Jw = ws.nj;
  const int ntree = blk ? (ws.na < B ? ws.na : B) : 0;
  // the solve's per-DOF arrays: slots of dofs_per_world per world (the world's
  // global DOF offset when the blocks are equal)
  const int n_slot = P.m.dofs_per_world;
  const size_t vs0 = (size_t)e * n_slot;
  double* poseA = reinterpret_cast<double*>(smem + L.pose);
  double* poseB = reinterpret_cast<double*>(smem + L.pose2);
  double* fm = reinterpret_cast<double*>(smem + L.fm);
  double* vj = reinterpret_cast<double*>(smem + L.vj);
  double* cbias = reinterpret_cast<double*>(smem + L.cb);
  double* vb = reinterpret_cast<double*>(smem + L.vb);
  double* fb = reinterpret_cast<double*>(smem + L.fb);
  double* ib = reinterpret_cast<double*>(smem + L.ib);
  double* fs = reinterpret_cast<double*>(smem + L.fs);
  double* S = reinterpret_cast<double*>(smem + L.S);
  double* Fi = reinterpret_cast<double*>(smem + L.F);
  double* tau = reinterpret_cast<double*>(smem + L.vec);
  double* vdot = tau + n;
  double* adiag = tau + 2 * n;
  double* dinv = tau + 3 * n;
  double* H = reinterpret_cast<double*>(smem + L.H);
  double* con = reinterpret_cast<double*>(smem + L.con);
  int* conint = reinterpret_cast<int*>(smem + L.conint);
  uint64_t* ancA = reinterpret_cast<uint64_t*>(smem + L.anc);
  uint64_t* ancB = ancA + B;
  int* jmpA = reinterpret_cast<int*>(smem + L.jmp);
  int* jmpB = jmpA + B;
  int* bj = reinterpret_cast<int*>(smem + L.bj);
  int* par = reinterpret_cast<int*>(smem + L.par);
  int* dbody = reinterpret_cast<int*>(smem + L.dbody);
  uint16_t* tri = reinterpret_cast<uint16_t*>(smem + L.tri);
  double* jg = reinterpret_cast<double*>(smem + L.jg);
  int* btree = reinterpret_cast<int*>(smem + L.trees);  // [B] tree of a body, -1
  int* tds = btree + B;                                  // [ntree + 1] first DOF of each tree
  const bool want_vstart = VS && !blk && P.out.v_start && P.gamma_start;
  const int j0 = ws.j0, b0g = ws.b0, d0 = ws.d0;
  const double* q = P.in.joint_q;
  const double* qd = P.in.joint_qd;

  // ---- topology of this world --------------------------------------------
  for (int b = tid; b < B; b += kPrepNT) {
    bj[b] = -1;
    if (blk) btree[b] = -1;
  }
  for (int i = tid; i < n; i += kPrepNT) dbody[i] = -1;
  if (!blk) build_triangle_list<kPrepNT>(tri, n);
  for (int k = tid; k < 6 * n; k += kPrepNT) S[k] = 0.0;
  if (want_vstart)
    for (int k = tid; k < (kPrepNT / 32) * n; k += kPrepNT) jg[k] = 0.0;
  // whether a live slot holds a new contact (the factor is then written
  // under factor_new_contacts_only)
  int newc = 0;
  if (P.o.factor_new_contacts_only && P.hist_depth) {
    const int tot = P.env_count[e];
    const int c0 = tot < C ? tot : C;
    for (int c = tid; c < c0; c += kPrepNT)
      if (P.hist_depth[(size_t)e * C + c] == 0) newc = 1;
  } else {
    newc = 1;
  }
  __syncthreads();
  for (int jl = tid; jl < Jw; jl += kPrepNT) {
    const int j = j0 + jl;
    const int cb = P.m.joint_child[j] - b0g;
    if (cb < 0 || cb >= B) continue;
    bj[cb] = j;
    const int dl = P.m.joint_qd_start[j] - d0;
    const int dim = P.m.joint_dof_dim[2 * j] + P.m.joint_dof_dim[2 * j + 1];
    for (int k = 0; k < dim; ++k)
      if (dl + k >= 0 && dl + k < n) dbody[dl + k] = cb;
  }
  // the trees of the tree-blocked outputs: the world's articulations, each a
  // contiguous DOF range
  for (int t = tid; t < ntree; t += kPrepNT) {
    const int ja = P.m.articulation_start[ws.a0 + t], jb = P.m.articulation_start[ws.a0 + t + 1];
    tds[t] = P.m.joint_qd_start[ja] - d0;
    if (t == ntree - 1) tds[ntree] = P.m.joint_qd_start[jb] - d0;
    for (int j = ja; j < jb; ++j) {
      const int cb = P.m.joint_child[j] - b0g;
      if (cb >= 0 && cb < B) btree[cb] = t;
    }
  }
  // (the barrier is unconditional: the topology and the tree starts above
  // are read across threads below)
  const bool write_factor = __syncthreads_or(newc) != 0 && P.out.dynamics_factor != nullptr;
  // a tree beyond the block size (or a broken articulation range): the
  // world's v* is NaN, which the solve reports as not finite
  bool tree_bad = false;
  if (blk) {
    bool bad = false;
    for (int t = tid; t < ntree; t += kPrepNT) {
      const int cnt = tds[t + 1] - tds[t];
      bad = bad || cnt < 0 || cnt > tb || tds[t] < 0 || tds[t + 1] > n;
    }
    tree_bad = __syncthreads_or(bad) != 0;
  }

  // ---- local transforms X_{parent body, body} = X_p X_FM(q) X_c^-1 ---------
  // (sim/sap_helpers.py:1164-1243)
  for (int b = tid; b < B; b += kPrepNT) {
    const int j = bj[b];
    Xf T{v3(0, 0, 0), qident()}, X_FM{v3(0, 0, 0), qident()};
    int parent = -1;
    if (j >= 0) {
      const int jt = P.m.joint_type[j];
      const int qs = P.m.joint_q_start[j], ds = P.m.joint_qd_start[j];
      if (jt == SAPB_JOINT_PRISMATIC) {
        X_FM.p = q[qs] * load3(P.m.joint_axis + 3 * (size_t)ds);
      } else if (jt == SAPB_JOINT_REVOLUTE) {
        X_FM.q = qaxis_angle(load3(P.m.joint_axis + 3 * (size_t)ds), q[qs]);
      } else if (jt == SAPB_JOINT_BALL) {
        X_FM.q = Q4{q[qs], q[qs + 1], q[qs + 2], q[qs + 3]};
      } else if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
        X_FM.p = v3(q[qs], q[qs + 1], q[qs + 2]);
        X_FM.q = Q4{q[qs + 3], q[qs + 4], q[qs + 5], q[qs + 6]};
      } else if (jt == SAPB_JOINT_D6) {
        V3 ax[3];
        d6_mobilizer(P.m.joint_axis + 3 * (size_t)ds, q + qs, P.m.joint_dof_dim[2 * j], P.m.joint_dof_dim[2 * j + 1],
                     &X_FM, ax);
      }
      T = xf_compose(xf_compose(xf_load(P.m.joint_X_p + 7 * (size_t)j), X_FM),
                     xf_inverse(xf_load(P.m.joint_X_c + 7 * (size_t)j)));
      parent = P.m.joint_parent[j] >= 0 ? P.m.joint_parent[j] - b0g : -1;
      if (parent >= B) parent = -1;
    }
    pose_store(poseA + 8 * b, T);
    pose_store(fm + 8 * b, X_FM);
    jmpA[b] = parent;
    par[b] = parent;
    ancA[b] = 1ull << b;
  }
  __syncthreads();
  // ---- world poses and ancestor masks by pointer jumping ------------------
  double* cur = poseA;
  double* nxt = poseB;
  int* jc = jmpA;
  int* jn = jmpB;
  uint64_t* ac = ancA;
  uint64_t* an = ancB;
  for (int round = 0; round < 8; ++round) {
    int active = 0;
    for (int b = tid; b < B; b += kPrepNT) {
      const int J = jc[b];
      if (J >= 0) {
        pose_store(nxt + 8 * b, xf_compose(pose_load(cur + 8 * J), pose_load(cur + 8 * b)));
        jn[b] = jc[J];
        an[b] = ac[b] | ac[J];
        active = 1;
      } else {
        for (int k = 0; k < 7; ++k) nxt[8 * b + k] = cur[8 * b + k];
        jn[b] = -1;
        an[b] = ac[b];
      }
    }
    double* t = cur;
    cur = nxt;
    nxt = t;
    int* tj = jc;
    jc = jn;
    jn = tj;
    uint64_t* ta = ac;
    ac = an;
    an = ta;
    if (!__syncthreads_or(active)) break;
  }
  const double* pose = cur;
  const uint64_t* anc = ac;
  // bodies by descending depth (children before their parents; equal depths
  // by index) for the subtree sums, in the pointer-jumping buffer left free
  int* deep_order = reinterpret_cast<int*>(an);

  // ---- motion subspaces, joint velocities, body inertias ------------------
  for (int b = tid; b < B; b += kPrepNT) {
    const int db = __popcll(anc[b]);  // depth + 1
    int rank = 0;
    for (int d = 0; d < B; ++d) {
      const int dd = __popcll(anc[d]);
      rank += (dd > db || (dd == db && d < b)) ? 1 : 0;
    }
    deep_order[rank] = b;
  }
  // S in world-origin coordinates of the reference's mobilizer columns
  // (sim/sap_helpers.py:1289-1433): revolute [w; p_F x w], prismatic [0; a],
  // ball [w_k; p_F x w_k], free [w_k; p_M x w_k] and [0; a_k], all axes
  // rotated by R_WF.
  const V3 grav = load3(P.m.gravity + 3 * (size_t)e);
  for (int b = tid; b < B; b += kPrepNT) {
    const int j = bj[b];
    Sv vJ = sv_zero(), c = sv_zero();
    if (j >= 0) {
      const int jt = P.m.joint_type[j];
      const int ds = P.m.joint_qd_start[j], dl = ds - d0;
      const int parent = P.m.joint_parent[j] >= 0 ? P.m.joint_parent[j] - b0g : -1;
      const Xf X_Wl = (parent >= 0 && parent < B) ? pose_load(pose + 8 * parent) : Xf{v3(0, 0, 0), qident()};
      const Xf X_WF = xf_compose(X_Wl, xf_load(P.m.joint_X_p + 7 * (size_t)j));
      const Xf X_WM = xf_compose(X_WF, pose_load(fm + 8 * b));
      const Q4 R = qnormalize(X_WF.q);
      auto put = [&](int k, Sv s) {
        sv_store(S + 6 * (dl + k), s);
        vJ = vJ + qd[ds + k] * s;
      };
      if (jt == SAPB_JOINT_PRISMATIC) {
        put(0, sv(v3(0, 0, 0), qrot(R, load3(P.m.joint_axis + 3 * (size_t)ds))));
      } else if (jt == SAPB_JOINT_REVOLUTE) {
        const V3 w = qrot(R, load3(P.m.joint_axis + 3 * (size_t)ds));
        put(0, sv(w, cross(X_WF.p, w)));
      } else if (jt == SAPB_JOINT_BALL) {
        for (int k = 0; k < 3; ++k) {
          const V3 w = qrot(R, v3(k == 0, k == 1, k == 2));
          put(k, sv(w, cross(X_WF.p, w)));
        }
      } else if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
        for (int k = 0; k < 3; ++k) {
          const V3 w = qrot(R, v3(k == 0, k == 1, k == 2));
          put(k, sv(w, cross(X_WM.p, w)));
          put(k + 3, sv(v3(0, 0, 0), w));
        }
        // the DOFs' own motion: d/dt of p_M x w_k along the relative
        // translation gives [0; v_rel x w_rel]
        const V3 w_rel = qrot(R, v3(qd[ds], qd[ds + 1], qd[ds + 2]));
        const V3 v_rel = qrot(R, v3(qd[ds + 3], qd[ds + 4], qd[ds + 5]));
        c = sv(v3(0, 0, 0), cross(v_rel, w_rel));
      } else if (jt == SAPB_JOINT_D6) {
        // translations [0; a_k], then rotations about M's origin [w_k; p_M x w_k]
        // (the rotation axes at the current angles, held fixed in the bias
        // like the reference, sim/sap_helpers.py:1387-1431)
        const int lin = P.m.joint_dof_dim[2 * j], ang = P.m.joint_dof_dim[2 * j + 1];
        Xf X_tmp;
        V3 ax[3];
        d6_mobilizer(P.m.joint_axis + 3 * (size_t)ds, q + P.m.joint_q_start[j], lin, ang, &X_tmp, ax);
        V3 v_rel = v3(0, 0, 0), w_rel = v3(0, 0, 0);
        for (int k = 0; k < lin && k < 3; ++k) {
          const V3 a = qrot(R, load3(P.m.joint_axis + 3 * (size_t)(ds + k)));
          put(k, sv(v3(0, 0, 0), a));
          v_rel = v_rel + qd[ds + k] * a;
        }
        for (int k = 0; k < ang && k < 3; ++k) {
          const V3 w = qrot(R, ax[k]);
          put(lin + k, sv(w, cross(X_WM.p, w)));
          w_rel = w_rel + qd[ds + lin + k] * w;
        }
        c = sv(v3(0, 0, 0), cross(v_rel, w_rel));
      }
    }
    sv_store(vj + 6 * b, vJ);
    sv_store(cbias + 6 * b, c);
    // inertia about the world origin (sim/sap_helpers.py:1027-1062)
    const Xf X = pose_load(pose + 8 * b);
    const Q4 qb = qnormalize(X.q);
    const double m = P.m.body_mass[b0g + b];
    const double* Ic = P.m.body_inertia + 9 * (size_t)(b0g + b);
    const V3 cw = X.p + qrot(qb, load3(P.m.body_com + 3 * (size_t)(b0g + b)));
    const V3 col[3] = {qrot(qb, v3(1, 0, 0)), qrot(qb, v3(0, 1, 0)), qrot(qb, v3(0, 0, 1))};
    const double Rm[3][3] = {{col[0].x, col[1].x, col[2].x}, {col[0].y, col[1].y, col[2].y},
                             {col[0].z, col[1].z, col[2].z}};
    double IW[3][3];
    for (int r = 0; r < 3; ++r)
      for (int t = 0; t < 3; ++t) {
        double acc = 0.0;
        for (int u = 0; u < 3; ++u)
          for (int v = 0; v < 3; ++v) acc += Rm[r][u] * Ic[3 * u + v] * Rm[t][v];
        IW[r][t] = acc;
      }
    const double cc = dot(cw, cw);
    double* I = ib + 10 * b;
    I[0] = m;
    I[1] = m * cw.x;
    I[2] = m * cw.y;
    I[3] = m * cw.z;
    I[4] = IW[0][0] + m * (cc - cw.x * cw.x);
    I[5] = IW[1][1] + m * (cc - cw.y * cw.y);
    I[6] = IW[2][2] + m * (cc - cw.z * cw.z);
    I[7] = IW[0][1] - m * cw.x * cw.y;
    I[8] = IW[0][2] - m * cw.x * cw.z;
    I[9] = IW[1][2] - m * cw.y * cw.z;
  }
  __syncthreads();
  // ---- body velocities: sums of the ancestors' joint velocities -------------
  for (int b = tid; b < B; b += kPrepNT) {
    Sv v = sv_zero();
    uint64_t mk = anc[b];
    while (mk) {
      const int d = __ffsll((long long)mk) - 1;
      mk &= mk - 1;
      v = v + sv_load(vj + 6 * d);
    }
    sv_store(vb + 6 * b, v);
  }
  __syncthreads();
  // joint bias accelerations c_b = v_parent x vJ_b (+ the free-joint term)
  for (int b = tid; b < B; b += kPrepNT) {
    const int j = bj[b];
    if (j < 0) continue;
    const int parent = P.m.joint_parent[j] >= 0 ? P.m.joint_parent[j] - b0g : -1;
    if (parent < 0 || parent >= B) continue;
    sv_store(cbias + 6 * b, sv_load(cbias + 6 * b) + crm(sv_load(vb + 6 * parent), sv_load(vj + 6 * b)));
  }
  __syncthreads();
  // ---- body forces f = I a + v x* I v - f_gravity + body_f -------------------
  // (sim/sap_helpers.py:1065-1105; gravity as the base acceleration -g)
  for (int b = tid; b < B; b += kPrepNT) {
    Sv a = sv(v3(0, 0, 0), -grav);
    uint64_t mk = anc[b];
    while (mk) {
      const int d = __ffsll((long long)mk) - 1;
      mk &= mk - 1;
      a = a + sv_load(cbias + 6 * d);
    }
    const double* I = ib + 10 * b;
    const Sv v = sv_load(vb + 6 * b);
    Sv f = inertia_times(I, a) + crf(v, inertia_times(I, v));
    if (P.in.body_f) {
      const Sv bf = sv_load(P.in.body_f + 6 * (size_t)(b0g + b));  // at the body origin
      const V3 pb = v3(pose[8 * b], pose[8 * b + 1], pose[8 * b + 2]);
      f = f + Sv{bf.w + cross(pb, bf.v), bf.v};
    }
    sv_store(fb + 6 * b, f);
  }
  __syncthreads();
  // ---- subtree forces and composite inertias: own values, then one pass
  // from the deepest bodies up, each adding its subtree into its parent
  for (int k = tid; k < 16 * B; k += kPrepNT) {
    const int b = k >> 4, comp = k & 15;
    fs[k] = comp < 6 ? fb[6 * b + comp] : ib[10 * b + comp - 6];
  }
  __syncthreads();
  for (int comp = tid; comp < 16; comp += kPrepNT) {
    for (int idx = 0; idx < B; ++idx) {
      const int b = deep_order[idx];
      const int p = par[b];
      if (p >= 0) fs[16 * p + comp] += fs[16 * b + comp];
    }
  }
  __syncthreads();
  // ---- tau = joint_f - S^T f_subtree, F_i = I^c S_i (sim/sap_helpers.py:2090-2118)
  for (int i = tid; i < n; i += kPrepNT) {
    const int b = dbody[i];
    Sv F = sv_zero();
    double t = P.in.joint_f ? P.in.joint_f[d0 + i] : 0.0;
    if (b >= 0) {
      const Sv s = sv_load(S + 6 * i);
      F = inertia_times(fs + 16 * b + 6, s);
      t -= sdot(s, sv_load(fs + 16 * b));
    }
    sv_store(Fi + 6 * i, F);
    tau[i] = t;
  }
  __syncthreads();
  // ---- A = composite-rigid-body pairs + armature ------------------------------
  if (blk) {
    // the tb x tb block of each tree (its DOFs tds[t] ..), the identity in
    // the padding of a tree with fewer DOFs
    const int bb = tb * tb;
    double* Tm = P.out.tree_mass + (size_t)e * ntree * bb;
    for (int k = tid; k < ntree * bb; k += kPrepNT) {
      const int t = k / bb, a = (k - t * bb) / tb, b = k % tb;
      const int s0 = tds[t], nt = tds[t + 1] - s0;
      double v = a == b ? 1.0 : 0.0;
      if (!tree_bad && a < nt && b < nt) {
        const int i = s0 + (a > b ? a : b), j = s0 + (a > b ? b : a);
        const int bi = dbody[i], bjj = dbody[j];
        v = 0.0;
        if (bi >= 0 && bjj >= 0) {
          if ((anc[bi] >> bjj) & 1ull) v = sdot(sv_load(S + 6 * j), sv_load(Fi + 6 * i));
          else if ((anc[bjj] >> bi) & 1ull) v = sdot(sv_load(S + 6 * i), sv_load(Fi + 6 * j));
        }
        if (a == b) {
          v += P.m.joint_armature[d0 + i];
          adiag[i] = v;
        }
      }
      H[k] = v;
      Tm[k] = v;
    }
  }
  double* Ag = blk ? nullptr : P.out.dynamics_matrix + (size_t)e * n_slot * n_slot;  // compact, stride n
  for (int k = tid; k < (blk ? 0 : n * n); k += kPrepNT) {
    const int i = k / n, j = k - i * n;
    if (j > i) continue;
    const int bi = dbody[i], bjj = dbody[j];
    double v = 0.0;
    if (bi >= 0 && bjj >= 0) {
      if ((anc[bi] >> bjj) & 1ull) v = sdot(sv_load(S + 6 * j), sv_load(Fi + 6 * i));
      else if ((anc[bjj] >> bi) & 1ull) v = sdot(sv_load(S + 6 * i), sv_load(Fi + 6 * j));
    }
    if (i == j) {
      v += P.m.joint_armature[d0 + i];
      adiag[i] = v;
    }
    H[(size_t)i * n + j] = v;
    Ag[(size_t)i * n + j] = v;
    Ag[(size_t)j * n + i] = v;
  }
  __syncthreads();

  // ---- free-motion solve A vdot = tau: LDL^T (H_ik = L_ik d_k below the diagonal)
  if (blk) {
    // a thread per tree: LDL^T of its block (its own DOFs; H_ab = L_ab d_b
    // below the diagonal, d on it) in place and the solve of its DOFs
    for (int t = tid; t < ntree; t += kPrepNT) {
      if (tree_bad) break;
      const int s0 = tds[t], nt = tds[t + 1] - s0;
      double* Ht = H + (size_t)t * tb * tb;
      for (int b = 0; b < nt; ++b) {
        double d = Ht[b * tb + b];
        for (int q = 0; q < b; ++q) d -= Ht[b * tb + q] * Ht[b * tb + q] * Ht[q * tb + q];
        Ht[b * tb + b] = d;
        const double r = 1.0 / d;
        for (int a = b + 1; a < nt; ++a) {
          double v = Ht[a * tb + b];
          for (int q = 0; q < b; ++q) v -= Ht[a * tb + q] * Ht[b * tb + q] * Ht[q * tb + q];
          Ht[a * tb + b] = v * r;
        }
      }
      double* z = vdot + s0;
      for (int a = 0; a < nt; ++a) {
        double v = tau[s0 + a];
        for (int q = 0; q < a; ++q) v -= Ht[a * tb + q] * z[q];
        z[a] = v;
      }
      for (int a = 0; a < nt; ++a) z[a] /= Ht[a * tb + a];
      for (int a = nt - 1; a >= 0; --a) {
        double v = z[a];
        for (int q = a + 1; q < nt; ++q) v -= Ht[q * tb + a] * z[q];
        z[a] = v;
      }
    }
  } else {
  ldlt_blocked<kPrepNT, double, 5>(H, n, n, dinv, tri);  // width 5: measured fastest for 35 DOFs
  if (write_factor) {
    double* Lg = P.out.dynamics_factor + (size_t)e * n_slot * n_slot;
    for (int k = tid; k < n * n; k += kPrepNT) {
      const int i = k / n, j = k - i * n;
      if (j <= i) Lg[k] = H[k];
    }
  }
  }
  // The free-motion solve A vdot = tau and the contact set-up below need
  // nothing of each other: with n <= 64, warp 0 solves by itself (shuffles,
  // no block barrier) while warps 1-3 rank and set up the contacts, synced by
  // a named barrier of their own; otherwise the whole block solves first.
  const bool split = !blk && n <= 64;
  if (!blk && !split) {
    for (int i = tid; i < n; i += kPrepNT) vdot[i] = tau[i];
    __syncthreads();
    ldlt_solve_blocked<kPrepNT, double>(H, n, n, dinv, vdot, false);
  }
  if (!split) __syncthreads();
  const int total = P.env_count[e];
  const int cc = total < C ? total : C;
  auto POSE_P = [&](int b) { return v3(pose[8 * b], pose[8 * b + 1], pose[8 * b + 2]); };
  auto POSE_Q = [&](int b) { return qnormalize(Q4{pose[8 * b + 3], pose[8 * b + 4], pose[8 * b + 5], pose[8 * b + 6]}); };
  if (split && tid < 32) {
    ldlt_solve_warp<double>(H, n, n, dinv, tau, vdot, false, ldlt_pivots_ok_warp<double>(H, n, n));
  } else {
  const int wt = split ? tid - 32 : tid;                // worker thread index
  const int wn = split ? kPrepNT - 32 : kPrepNT;        // worker threads
  auto wsync = [&]() {
    if (split) asm volatile("bar.sync 1, %0;" ::"n"(kPrepNT - 32) : "memory");
    else __syncthreads();
  };
  // ---- contacts of this world ---------------------------------------------
  if (wt == 0 && P.out.contact_count) P.out.contact_count[e] = total;
  // Canonical slot order: the slots the scatter claimed in arrival order are
  // re-ranked by flat contact index (distinct), so an untruncated world's
  // slots follow the flat buffer's order on every step.
  if (!P.ranked) {  // (the contact history ranks them when it runs first)
    int* tmp = conint;  // 2*C ints, free until the rows below use them
    for (int c = wt; c < cc; c += wn) tmp[c] = P.env_src[(size_t)e * C + c];
    wsync();
    for (int c = wt; c < cc; c += wn) {
      const int v = tmp[c];
      int rank = 0;
      for (int j = 0; j < cc; ++j) rank += tmp[j] < v ? 1 : 0;
      P.env_src[(size_t)e * C + rank] = v;
    }
    wsync();
  }
  if (P.out.contact_source)
    for (int c = wt; c < C; c += wn) P.out.contact_source[(size_t)e * C + c] = c < cc ? P.env_src[(size_t)e * C + c] : -1;
  for (int c = wt; c < cc; c += wn) {
    const int src = P.env_src[(size_t)e * C + c];
    const int sh0 = P.in.contact_shape0[src], sh1 = P.in.contact_shape1[src];
    const int S_ = P.m.num_shapes;
    const int gb0 = (sh0 >= 0 && sh0 < S_) ? P.m.shape_body[sh0] : -1;
    const int gb1 = (sh1 >= 0 && sh1 < S_) ? P.m.shape_body[sh1] : -1;
    const int lb0 = gb0 >= 0 ? gb0 - b0g : -1, lb1 = gb1 >= 0 ? gb1 - b0g : -1;
    V3 x0 = load3(P.in.contact_point0 + 3 * (size_t)src);
    V3 x1 = load3(P.in.contact_point1 + 3 * (size_t)src);
    if (lb0 >= 0) x0 = POSE_P(lb0) + qrot(POSE_Q(lb0), x0);
    if (lb1 >= 0) x1 = POSE_P(lb1) + qrot(POSE_Q(lb1), x1);
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
    double* cs = con + kConStride * (size_t)c;
    const bool mid = P.o.contact_point_mode == SAPB_POINT_MIDPOINT;
    store3(cs + 0, mid ? pC : x0);
    store3(cs + 3, mid ? pC : x1);
    for (int k = 0; k < 9; ++k) cs[kConFrame + k] = F[k];
    conint[2 * c] = (lb0 >= 0 && lb0 < B) ? lb0 : -1;
    conint[2 * c + 1] = (lb1 >= 0 && lb1 < B) ? lb1 : -1;
  }
  }
  __syncthreads();
  for (int i = tid; i < n; i += kPrepNT) {
    const double vd = vdot[i];
    P.out.v_star[vs0 + i] = tree_bad ? __longlong_as_double(0x7ff8000000000000ll)
                                     : P.in.joint_qd[d0 + i] + P.in.dt[e] * vd;
    if (P.out.vdot) P.out.vdot[vs0 + i] = vd;
    if (P.out.qd_slots) P.out.qd_slots[vs0 + i] = P.in.joint_qd[d0 + i];
  }
  if (P.out.body_q) {
    for (int k = tid; k < 7 * B; k += kPrepNT) {
      const int b = k / 7, c = k - 7 * b;
      P.out.body_q[7 * (size_t)(b0g + b) + c] = pose[8 * b + c];
    }
  }
  // ---- contact rows, free-motion contact velocities and diag_delassus
  // weights, one warp per contact: lanes over the DOF columns, row / weight
  // partial sums reduced by shuffles.
  // Tree-blocked rows hold 2 tb columns: the tb columns of side 0's tree
  // (zero beyond its own DOFs), then side 1's (a contact between two shapes
  // of one tree keeps the combined columns on side 0).
  const int ncols = blk ? 2 * tb : n;
  double* Jout = P.out.jacobian + (size_t)e * C * 3 * (blk ? 2 * tb : n_slot);  // rows compact, stride ncols
  auto tree_of = [&](int lb) { return lb < 0 ? -1 : btree[lb]; };
  {
    const int lane = tid & 31, warp = tid >> 5;
    const bool dd = P.o.contact_weight_mode == SAPB_WEIGHT_DIAG_DELASSUS;
    // this warp's partial of J^T gamma_start (its contacts, in order): in
    // registers, columns lane and lane + 32, up to 64 DOFs; in shared memory beyond
    double jgr0 = 0.0, jgr1 = 0.0;
    const double h = P.in.dt[e];
    for (int c = warp; c < cc; c += kPrepNT / 32) {
      const double* cs = con + kConStride * (size_t)c;
      const int lb0 = conint[2 * c], lb1 = conint[2 * c + 1];
      int t0 = -1, t1 = -1;
      if (blk) {
        t0 = tree_of(lb0);
        t1 = tree_of(lb1);
        if (t1 == t0) t1 = -1;
        if (t0 < 0) {
          t0 = t1;
          t1 = -1;
        }
        if (lane == 0) {
          // the side order of the rows: the body of side 0 (or the only one)
          P.out.contact_tree[2 * ((size_t)e * C + c)] = t0;
          P.out.contact_tree[2 * ((size_t)e * C + c) + 1] = t1;
        }
      }
      double wq[6] = {0, 0, 0, 0, 0, 0}, vq[3] = {0, 0, 0};
      const double* gst = want_vstart ? P.gamma_start + 3 * ((size_t)e * C + c) : nullptr;
      for (int col = lane; col < ncols; col += 32) {
        V3 rel = v3(0, 0, 0);
        int dof = col;
        if (blk) {
          const int ts = col < tb ? t0 : t1, a = col < tb ? col : col - tb;
          dof = (ts >= 0 && !tree_bad && a < tds[ts + 1] - tds[ts]) ? tds[ts] + a : -1;
        }
        const int bcol = dof >= 0 ? dbody[dof] : -1;
        if (bcol >= 0) {
          const Sv sc = sv_load(S + 6 * dof);
          if (lb1 >= 0 && ((anc[lb1] >> bcol) & 1ull)) rel = rel + (sc.v + cross(sc.w, load3(cs + 3)));
          if (lb0 >= 0 && ((anc[lb0] >> bcol) & 1ull)) rel = rel - (sc.v + cross(sc.w, load3(cs + 0)));
        }
        double rw[3];
        for (int r = 0; r < 3; ++r) {
          rw[r] = dot(load3(cs + kConFrame + 3 * r), rel);
          Jout[((size_t)c * 3 + r) * ncols + col] = rw[r];
        }
        if (dof < 0) continue;
        if (want_vstart) {
          const double t = rw[0] * __ldg(gst) + rw[1] * __ldg(gst + 1) + rw[2] * __ldg(gst + 2);
          if (n <= 64) {
            if (col < 32) jgr0 += t;
            else jgr1 += t;
          } else {
            jg[warp * n + dof] += t;
          }
        }
        const double vs = P.in.joint_qd[d0 + dof] + h * vdot[dof];
        vq[0] += rw[0] * vs;
        vq[1] += rw[1] * vs;
        vq[2] += rw[2] * vs;
        if (dd) {
          double aii = adiag[dof];
          if (aii < 1.0e-12) aii = 1.0e-12;
          const double inv = 1.0 / aii;
          wq[0] += inv * rw[0] * rw[0];
          wq[1] += inv * rw[0] * rw[1];
          wq[2] += inv * rw[0] * rw[2];
          wq[3] += inv * rw[1] * rw[1];
          wq[4] += inv * rw[1] * rw[2];
          wq[5] += inv * rw[2] * rw[2];
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) vq[k] += __shfl_xor_sync(0xffffffffu, vq[k], o);
        if (dd) {
#pragma unroll
          for (int k = 0; k < 6; ++k) wq[k] += __shfl_xor_sync(0xffffffffu, wq[k], o);
        }
      }
      if (lane == 0) {
        const size_t ci = (size_t)e * C + c;
        if (P.out.vc_star)
          for (int k = 0; k < 3; ++k) P.out.vc_star[3 * ci + k] = vq[k];
        if (dd) {
          // ||J diag(A)^-1 J^T||_F / 3 (sim/contact_jacobian.py:153-251)
          const double wv = sqrt(wq[0] * wq[0] + wq[3] * wq[3] + wq[5] * wq[5] +
                                 2.0 * (wq[1] * wq[1] + wq[2] * wq[2] + wq[4] * wq[4])) / 3.0;
          P.out.w_eff[ci] = wv < 1.0e-12 ? 1.0e-12 : wv;
        }
      }
    }
    if (want_vstart && n <= 64) {
      if (lane < n) jg[warp * n + lane] = jgr0;
      if (lane + 32 < n) jg[warp * n + lane + 32] = jgr1;
    }
  }
  __syncthreads();
  // ---- body_inertia contact weights (sim/contact_jacobian.py:153-251) --------
  if (P.o.contact_weight_mode != SAPB_WEIGHT_DIAG_DELASSUS) {
  for (int c = tid; c < cc; c += kPrepNT) {
    const size_t ci = (size_t)e * C + c;
    double w = 0.0;
    {
      const double* cs = con + kConStride * (size_t)c;
      const int lbs[2] = {conint[2 * c], conint[2 * c + 1]};
      // body-inertia weights use the witnesses, whatever the point mode
      const int src = P.env_src[ci];
      double wsum = 0.0;
      for (int side = 0; side < 2; ++side) {
        const int lb = lbs[side];
        if (lb < 0) continue;
        const double mass = P.m.body_mass[b0g + lb];
        if (mass <= 1.0e-12) continue;
        const Q4 qq = POSE_Q(lb);
        const V3 pb = POSE_P(lb);
        const V3 xw = pb + qrot(qq, load3((side == 0 ? P.in.contact_point0 : P.in.contact_point1) + 3 * (size_t)src));
        const V3 com = pb + qrot(qq, load3(P.m.body_com + 3 * (size_t)(b0g + lb)));
        const V3 r = xw - com;
        const double* Ic = P.m.body_inertia + 9 * (size_t)(b0g + lb);
        const double ix = fmax(Ic[0], 1.0e-12), iy = fmax(Ic[4], 1.0e-12), iz = fmax(Ic[8], 1.0e-12);
        for (int d = 0; d < 3; ++d) {
          const V3 cb = qrot(qconj(qq), cross(r, load3(cs + kConFrame + 3 * d)));
          wsum += 1.0 / mass + cb.x * cb.x / ix + cb.y * cb.y / iy + cb.z * cb.z / iz;
        }
      }
      w = wsum / 3.0;
    }
    P.out.w_eff[ci] = w < 1.0e-12 ? 1.0e-12 : w;
  }
  }
  // ---- candidate start v* + A^-1 J^T gamma_start through this kernel's
  // LDL^T of A (H, dinv): the warps' partials summed in warp order, then the
  // triangular solves (one warp up to 64 DOFs, the block beyond)
  if (want_vstart && n <= 64) {
    __syncthreads();
    if (tid < 32) {  // warp 0 alone: no block barrier after the partials
      double* z = jg + n;
      for (int i = tid; i < n; i += 32) {
        double r = 0.0;
        for (int q = 0; q < kPrepNT / 32; ++q) r += jg[q * n + i];
        jg[i] = r;
      }
      __syncwarp();
      ldlt_solve_warp<double>(H, n, n, dinv, jg, z, false, ldlt_pivots_ok_warp<double>(H, n, n));
      __syncwarp();
      for (int i = tid; i < n; i += 32)
        P.out.v_start[vs0 + i] = P.in.joint_qd[d0 + i] + P.in.dt[e] * vdot[i] + z[i];
    }
  } else if (want_vstart) {
    __syncthreads();
    for (int i = tid; i < n; i += kPrepNT) {
      double r = 0.0;
      for (int q = 0; q < kPrepNT / 32; ++q) r += jg[q * n + i];
      jg[i] = r;
    }
    __syncthreads();
    double* z = jg + n;
    {
      for (int i = tid; i < n; i += kPrepNT) z[i] = jg[i];
      __syncthreads();
      ldlt_solve_blocked<kPrepNT, double>(H, n, n, dinv, z, false);
    }
    __syncthreads();
    for (int i = tid; i < n; i += kPrepNT)
      P.out.v_start[vs0 + i] = P.in.joint_qd[d0 + i] + P.in.dt[e] * vdot[i] + z[i];
  }
}

size_t prepare_smem_bytes(int B, int n, int C, int tree_block) { return prep_layout(B, n, C, tree_block).total; }

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
  if (err == cudaSuccess && out->history) {
    // the contact history on this launch's slots, which it ranks by flat index
    sapb_contact_history hh = *out->history;
    hh.num_envs = W;
    hh.max_contacts = C > 0 ? C : 1;
    hh.num_flat = in->contact_capacity;
    hh.contact_count = P.env_count;
    hh.contact_source = nullptr;
    hh.flat_shape0 = in->contact_shape0;
    hh.flat_shape1 = in->contact_shape1;
    hh.flat_point1 = in->contact_point1;
    const int32_t st = history_launch(&hh, P.env_src, stream);
    if (st != SAPB_OK) return st;
    P.ranked = true;
    P.gamma_start = hh.gamma_start;
    P.hist_depth = hh.has_history;
  }
  if (err == cudaSuccess) {
    const int tree_block = o->tree_blocked ? (o->tree_dofs > 0 ? o->tree_dofs : 6) : 0;
    const size_t smem = prepare_smem_bytes(m->bodies_per_world, m->dofs_per_world, C, tree_block);
    const bool vs = out->v_start && P.gamma_start && !o->tree_blocked;
    err = cudaFuncSetAttribute(vs ? prepare_world_kernel<true> : prepare_world_kernel<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err == cudaSuccess) {
      if (vs) prepare_world_kernel<true><<<W, kPrepNT, smem, stream>>>(P);
      else prepare_world_kernel<false><<<W, kPrepNT, smem, stream>>>(P);
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
  integrate_joint(m, j, q_in, v_prev, v_new, dt[j / m.joints_per_world], mode, q_out);
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
