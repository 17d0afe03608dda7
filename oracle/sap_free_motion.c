/*
 * sap_free_motion.c -- C restatement of the reference's free motion, contact
 * Jacobian and position integration -- TEST INFRASTRUCTURE ONLY (the checker
 * for the CUDA free-motion kernel and the CPU pipeline timed beside the GPU).
 *
 * Same descriptor structs as the device entry points (include/sapb.h) with
 * HOST pointers.  The recursions are the reference's body-origin ones (joint
 * by joint, spatial vectors [angular; linear] at the body origin in world
 * coordinates, sim/sap_helpers.py:771-785), independent of the GPU kernel's
 * world-origin formulation; oracle/free_motion.py is the same algorithm in
 * numpy.  Worlds run in parallel with OpenMP.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "sap_oracle.h"

typedef struct {
  double x, y, z;
} v3_t;
typedef struct {
  double x, y, z, w;
} q4_t;
typedef struct {
  v3_t p;
  q4_t q;
} xf_t;

static v3_t v3(double x, double y, double z) {
  v3_t r = {x, y, z};
  return r;
}
static v3_t vadd(v3_t a, v3_t b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3_t vsub(v3_t a, v3_t b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3_t vscale(double s, v3_t a) { return v3(s * a.x, s * a.y, s * a.z); }
static double dot3(v3_t a, v3_t b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3_t vcross(v3_t a, v3_t b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3_t vload(const double* p) { return v3(p[0], p[1], p[2]); }
static void vstore(double* p, v3_t a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

/* quaternions xyzw and transforms (sim/sap_helpers.py:576-700) */
static q4_t qmul(q4_t a, q4_t b) {
  q4_t r = {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
  return r;
}
static q4_t qnorm(q4_t q) {
  const double n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q4_t id = {0, 0, 0, 1};
  if (!(n > 0.0)) return id;
  q4_t r = {q.x / n, q.y / n, q.z / n, q.w / n};
  return r;
}
static q4_t qconj(q4_t q) {
  q4_t r = {-q.x, -q.y, -q.z, q.w};
  return r;
}
static v3_t qrot(q4_t q, v3_t v) {
  const v3_t qv = v3(q.x, q.y, q.z);
  const v3_t t = vscale(2.0, vcross(qv, v));
  return vadd(vadd(v, vscale(q.w, t)), vcross(qv, t));
}
static q4_t qaxis(v3_t a, double angle) {
  const double h = 0.5 * angle, s = sin(h);
  q4_t r = {a.x * s, a.y * s, a.z * s, cos(h)};
  return r;
}
static xf_t xload(const double* p) {
  xf_t x = {v3(p[0], p[1], p[2]), {p[3], p[4], p[5], p[6]}};
  return x;
}
static xf_t xcompose(xf_t a, xf_t b) {
  const q4_t aq = qnorm(a.q), bq = qnorm(b.q);
  xf_t r = {vadd(a.p, qrot(aq, b.p)), qnorm(qmul(aq, bq))};
  return r;
}
static xf_t xinverse(xf_t x) {
  const q4_t qi = qconj(qnorm(x.q));
  xf_t r = {vscale(-1.0, qrot(qi, x.p)), qi};
  return r;
}

/* spatial vectors [w; v] (sim/sap_helpers.py:862-1024) */
typedef struct {
  v3_t w, v;
} sv_t;
static sv_t sv(v3_t w, v3_t v) {
  sv_t r = {w, v};
  return r;
}
static sv_t sload(const double* p) { return sv(vload(p), vload(p + 3)); }
static void sstore(double* p, sv_t a) {
  vstore(p, a.w);
  vstore(p + 3, a.v);
}
static double sdot(sv_t a, sv_t b) { return dot3(a.w, b.w) + dot3(a.v, b.v); }
static sv_t shift_velocity(sv_t V, v3_t p) { return sv(V.w, vadd(V.v, vcross(V.w, p))); }
static sv_t shift_acceleration(sv_t A, v3_t p, v3_t w) {
  return sv(A.w, vadd(vadd(A.v, vcross(A.w, p)), vcross(w, vcross(w, p))));
}
static sv_t shift_force(sv_t F, v3_t p) { return sv(vsub(F.w, vcross(p, F.v)), F.v); }
static sv_t compose_velocity(sv_t Vp, v3_t p, sv_t Vpb) {
  return sv(vadd(Vp.w, Vpb.w), vadd(vadd(Vp.v, vcross(Vp.w, p)), Vpb.v));
}
static sv_t compose_acceleration(sv_t Ap, sv_t Vp, v3_t p, sv_t Vpb, sv_t Apb) {
  const v3_t w = Vp.w;
  const sv_t As = shift_acceleration(Ap, p, w);
  return sv(vadd(vadd(As.w, Apb.w), vcross(w, Vpb.w)), vadd(vadd(As.v, Apb.v), vscale(2.0, vcross(w, Vpb.v))));
}
static sv_t mob_velocity(q4_t R, v3_t p, sv_t Vfm) {
  return sv(qrot(R, Vfm.w), qrot(R, vadd(Vfm.v, vcross(Vfm.w, p))));
}
static sv_t mob_bias(q4_t R, v3_t p, v3_t w) { return sv(v3(0, 0, 0), qrot(R, vcross(w, vcross(w, p)))); }

/* rows t1, t2, n of _sap_make_from_one_unit_vector_z (sim/sap_helpers.py:467-503) */
static void contact_frame(v3_t n, double F[9]) {
  const double a[3] = {fabs(n.x), fabs(n.y), fabs(n.z)};
  int i = 0;
  double mn = a[0];
  if (a[1] < mn) {
    i = 1;
    mn = a[1];
  }
  if (a[2] < mn) {
    i = 2;
    mn = a[2];
  }
  const double mag = sqrt(1.0 - mn * mn), r = 1.0 / mag;
  const double umin = i == 0 ? n.x : (i == 1 ? n.y : n.z);
  const double s = -r * umin;
  v3_t v, w;
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
  vstore(F, v);
  vstore(F + 3, w);
  vstore(F + 6, n);
}

/* material fallbacks (sim/sap_helpers.py:150-237) */
static double mat_mu(const sapb_model_desc* m, const sapb_prepare_options* o, int sh) {
  double v = o->fallback_mu;
  if (sh >= 0 && m->shape_material_mu) v = m->shape_material_mu[sh];
  return v < 0.0 ? 0.0 : v;
}
static double mat_k(const sapb_model_desc* m, const sapb_prepare_options* o, int sh) {
  double v = o->fallback_stiffness;
  if (sh >= 0 && m->shape_material_ke) v = m->shape_material_ke[sh];
  if (!isfinite(v) || v <= 0.0) v = o->fallback_stiffness;
  if (!isfinite(v) || v <= 0.0) v = 1.0;
  return v;
}
static double mat_tau(const sapb_model_desc* m, const sapb_prepare_options* o, int sh) {
  double v = o->fallback_tau_d;
  if (sh >= 0 && m->shape_material_tau) v = m->shape_material_tau[sh];
  if (!isfinite(v) || v < 0.0) v = o->fallback_tau_d;
  if (!isfinite(v) || v < 0.0) v = 0.0;
  return v;
}

static void world_step(const sapb_model_desc* m, const sapb_step_inputs* in, const sapb_prepare_options* o,
                       const sapb_prepare_outputs* out, const int32_t* slot_src, const int32_t* world_total, int e) {
  const int B = m->bodies_per_world, Jw = m->joints_per_world, n = m->dofs_per_world, C = o->max_contacts;
  const int j0 = e * Jw, b0g = e * B, d0 = e * n;
  double* pose = (double*)calloc((size_t)B * 7, sizeof(double));
  double* V = (double*)calloc((size_t)B * 6, sizeof(double));
  double* Ab = (double*)calloc((size_t)B * 6, sizeof(double));
  double* S = (double*)calloc((size_t)n * 6, sizeof(double));
  double* I6 = (double*)calloc((size_t)B * 36, sizeof(double));
  double* fbody = (double*)calloc((size_t)B * 6, sizeof(double));
  double* ft = (double*)calloc((size_t)B * 6, sizeof(double));
  double* tau = (double*)calloc((size_t)n, sizeof(double));
  double* Jb = (double*)calloc((size_t)B * 6 * n, sizeof(double));
  double* A = (double*)calloc((size_t)n * n, sizeof(double));
  double* L = (double*)calloc((size_t)n * n, sizeof(double));
  double* vdot = (double*)calloc((size_t)n, sizeof(double));
  for (int b = 0; b < B; ++b) pose[7 * b + 6] = 1.0;
  const double* q = in->joint_q;
  const double* qd = in->joint_qd;

  /* FK, velocities, bias accelerations (sim/free_motion.py:412-530, sim/sap_helpers.py:1164-1433) */
  for (int jl = 0; jl < Jw; ++jl) {
    const int j = j0 + jl;
    const int jt = m->joint_type[j];
    const int lp = m->joint_parent[j] >= 0 ? m->joint_parent[j] - b0g : -1;
    const int lc = m->joint_child[j] - b0g;
    const int qs = m->joint_q_start[j], ds = m->joint_qd_start[j], dl = ds - d0;
    const xf_t Xp = xload(m->joint_X_p + 7 * (size_t)j), Xc = xload(m->joint_X_c + 7 * (size_t)j);
    xf_t X_WF = Xp;
    if (lp >= 0) X_WF = xcompose(xload(pose + 7 * lp), Xp);
    xf_t X_FM = {v3(0, 0, 0), {0, 0, 0, 1}};
    sv_t V_FM = sv(v3(0, 0, 0), v3(0, 0, 0));
    const v3_t ax = vload(m->joint_axis + 3 * (size_t)ds);
    int dim = 0;
    if (jt == SAPB_JOINT_PRISMATIC) {
      X_FM.p = vscale(q[qs], ax);
      V_FM = sv(v3(0, 0, 0), vscale(qd[ds], ax));
      dim = 1;
    } else if (jt == SAPB_JOINT_REVOLUTE) {
      X_FM.q = qaxis(ax, q[qs]);
      V_FM = sv(vscale(qd[ds], ax), v3(0, 0, 0));
      dim = 1;
    } else if (jt == SAPB_JOINT_BALL) {
      q4_t qq = {q[qs], q[qs + 1], q[qs + 2], q[qs + 3]};
      X_FM.q = qq;
      V_FM = sv(v3(qd[ds], qd[ds + 1], qd[ds + 2]), v3(0, 0, 0));
      dim = 3;
    } else if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
      q4_t qq = {q[qs + 3], q[qs + 4], q[qs + 5], q[qs + 6]};
      X_FM.p = v3(q[qs], q[qs + 1], q[qs + 2]);
      X_FM.q = qq;
      V_FM = sv(v3(qd[ds], qd[ds + 1], qd[ds + 2]), v3(qd[ds + 3], qd[ds + 4], qd[ds + 5]));
      dim = 6;
    }
    const xf_t X_WM = xcompose(X_WF, X_FM);
    const xf_t X_MB = xinverse(Xc);
    const xf_t X_WB = xcompose(X_WM, X_MB);
    const v3_t p = qrot(qnorm(X_FM.q), X_MB.p);
    const q4_t R = qnorm(X_WF.q);
    if (jt == SAPB_JOINT_PRISMATIC) {
      sstore(S + 6 * dl, mob_velocity(R, p, sv(v3(0, 0, 0), ax)));
    } else if (jt == SAPB_JOINT_REVOLUTE) {
      sstore(S + 6 * dl, sv(qrot(R, ax), qrot(R, vcross(ax, p))));
    } else if (dim == 3 || dim == 6) {
      for (int k = 0; k < dim; ++k) {
        double u[6] = {0, 0, 0, 0, 0, 0};
        u[k] = 1.0;
        sstore(S + 6 * (dl + k), mob_velocity(R, p, sload(u)));
      }
    }
    const sv_t Vpb = dim > 0 ? mob_velocity(R, p, V_FM) : sv(v3(0, 0, 0), v3(0, 0, 0));
    const sv_t Apb = dim > 0 ? mob_bias(R, p, V_FM.w) : sv(v3(0, 0, 0), v3(0, 0, 0));
    vstore(pose + 7 * lc, X_WB.p);
    pose[7 * lc + 3] = X_WB.q.x;
    pose[7 * lc + 4] = X_WB.q.y;
    pose[7 * lc + 5] = X_WB.q.z;
    pose[7 * lc + 6] = X_WB.q.w;
    if (lp >= 0) {
      const sv_t Vp = sload(V + 6 * lp), Ap = sload(Ab + 6 * lp);
      const v3_t pPB = vsub(X_WB.p, vload(pose + 7 * lp));
      sstore(V + 6 * lc, compose_velocity(Vp, pPB, Vpb));
      sstore(Ab + 6 * lc, compose_acceleration(Ap, Vp, pPB, Vpb, Apb));
    } else {
      sstore(V + 6 * lc, Vpb);
      sstore(Ab + 6 * lc, Apb);
    }
  }
  /* body dynamics (sim/free_motion.py:680-719, sim/sap_helpers.py:1027-1105) */
  const v3_t g = vload(m->gravity + 3 * (size_t)e);
  for (int b = 0; b < B; ++b) {
    const q4_t qb = qnorm(*(const q4_t*)(pose + 7 * b + 3));
    const double mass = m->body_mass[b0g + b];
    const double* Ic = m->body_inertia + 9 * (size_t)(b0g + b);
    double R[3][3];
    for (int c = 0; c < 3; ++c) {
      const v3_t col = qrot(qb, v3(c == 0, c == 1, c == 2));
      R[0][c] = col.x;
      R[1][c] = col.y;
      R[2][c] = col.z;
    }
    const v3_t c = qrot(qb, vload(m->body_com + 3 * (size_t)(b0g + b)));
    const double cc[3] = {c.x, c.y, c.z};
    double* I = I6 + 36 * b;
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        double acc = 0.0;
        for (int u = 0; u < 3; ++u)
          for (int v = 0; v < 3; ++v) acc += R[r][u] * Ic[3 * u + v] * R[s][v];
        I[6 * r + s] = acc + mass * ((r == s ? dot3(c, c) : 0.0) - cc[r] * cc[s]);
        I[6 * (r + 3) + (s + 3)] = r == s ? mass : 0.0;
      }
    const double cx[3][3] = {{0.0, -c.z, c.y}, {c.z, 0.0, -c.x}, {-c.y, c.x, 0.0}};
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        I[6 * r + (s + 3)] = mass * cx[r][s];
        I[6 * (r + 3) + s] = -mass * cx[r][s];
      }
    const double* a = Ab + 6 * b;
    double f[6];
    for (int r = 0; r < 6; ++r) {
      double acc = 0.0;
      for (int s = 0; s < 6; ++s) acc += I[6 * r + s] * a[s];
      f[r] = acc;
    }
    const v3_t w = vload(V + 6 * b);
    const v3_t Iw = v3(I[0] * w.x + I[1] * w.y + I[2] * w.z, I[6] * w.x + I[7] * w.y + I[8] * w.z,
                       I[12] * w.x + I[13] * w.y + I[14] * w.z);
    const v3_t bt = vcross(w, Iw), bf = vscale(mass, vcross(w, vcross(w, c)));
    const v3_t fg = vscale(mass, g), tg = vcross(c, fg);
    double* fb = fbody + 6 * b;
    fb[0] = f[0] + bt.x - tg.x;
    fb[1] = f[1] + bt.y - tg.y;
    fb[2] = f[2] + bt.z - tg.z;
    fb[3] = f[3] + bf.x - fg.x;
    fb[4] = f[4] + bf.y - fg.y;
    fb[5] = f[5] + bf.z - fg.z;
  }
  /* reverse pass (sim/free_motion.py:154-220, sim/sap_helpers.py:2090-2118) */
  for (int jl = Jw - 1; jl >= 0; --jl) {
    const int j = j0 + jl;
    const int lp = m->joint_parent[j] >= 0 ? m->joint_parent[j] - b0g : -1;
    const int lc = m->joint_child[j] - b0g;
    const int ds = m->joint_qd_start[j], dl = ds - d0;
    const int dim = m->joint_dof_dim[2 * j] + m->joint_dof_dim[2 * j + 1];
    sv_t fs = sv(vadd(vload(fbody + 6 * lc), vload(ft + 6 * lc)), vadd(vload(fbody + 6 * lc + 3), vload(ft + 6 * lc + 3)));
    if (in->body_f) {
      const sv_t bfx = sload(in->body_f + 6 * (size_t)(b0g + lc));
      fs = sv(vadd(fs.w, bfx.w), vadd(fs.v, bfx.v));
    }
    for (int k = 0; k < dim; ++k)
      tau[dl + k] = -sdot(sload(S + 6 * (dl + k)), fs) + (in->joint_f ? in->joint_f[ds + k] : 0.0);
    if (lp >= 0) {
      const sv_t sf = shift_force(fs, vsub(vload(pose + 7 * lp), vload(pose + 7 * lc)));
      double* t = ft + 6 * lp;
      t[0] += sf.w.x;
      t[1] += sf.w.y;
      t[2] += sf.w.z;
      t[3] += sf.v.x;
      t[4] += sf.v.y;
      t[5] += sf.v.z;
    }
  }
  /* body Jacobians (sim/free_motion.py:722-765) and A = sum J^T I J + armature (:814-1179) */
  for (int jl = 0; jl < Jw; ++jl) {
    const int j = j0 + jl;
    const int lc = m->joint_child[j] - b0g;
    for (int jj = j; jj >= 0; jj = m->joint_ancestor[jj]) {
      const int cb = m->joint_child[jj] - b0g;
      const int dl = m->joint_qd_start[jj] - d0;
      const int dim = m->joint_dof_dim[2 * jj] + m->joint_dof_dim[2 * jj + 1];
      const v3_t pp = vsub(vload(pose + 7 * lc), vload(pose + 7 * cb));
      for (int k = 0; k < dim; ++k) {
        double o6[6];
        sstore(o6, shift_velocity(sload(S + 6 * (dl + k)), pp));
        for (int r = 0; r < 6; ++r) Jb[((size_t)lc * 6 + r) * n + dl + k] = o6[r];
      }
    }
  }
  for (int b = 0; b < B; ++b) {
    const double* I = I6 + 36 * b;
    const double* J = Jb + (size_t)b * 6 * n;
    for (int jc = 0; jc < n; ++jc) {
      double k6[6];
      for (int r = 0; r < 6; ++r) {
        double acc = 0.0;
        for (int s = 0; s < 6; ++s) acc += I[6 * r + s] * J[(size_t)s * n + jc];
        k6[r] = acc;
      }
      for (int ic = jc; ic < n; ++ic) {
        double acc = 0.0;
        for (int r = 0; r < 6; ++r) acc += J[(size_t)r * n + ic] * k6[r];
        A[(size_t)ic * n + jc] += acc;
      }
    }
  }
  for (int i = 0; i < n; ++i) {
    A[(size_t)i * n + i] += m->joint_armature[d0 + i];
    for (int j = i + 1; j < n; ++j) A[(size_t)i * n + j] = A[(size_t)j * n + i];
  }
  memcpy(L, A, sizeof(double) * (size_t)n * n);
  sapo_cholesky(L, n);
  for (int i = 0; i < n; ++i) {
    double t = tau[i];
    for (int k = 0; k < i; ++k) t -= L[(size_t)i * n + k] * vdot[k];
    vdot[i] = t / L[(size_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double t = vdot[i];
    for (int k = i + 1; k < n; ++k) t -= L[(size_t)k * n + i] * vdot[k];
    vdot[i] = t / L[(size_t)i * n + i];
  }
  const double h = in->dt[e];
  memcpy(out->dynamics_matrix + (size_t)e * n * n, A, sizeof(double) * (size_t)n * n);
  for (int i = 0; i < n; ++i) {
    out->v_star[d0 + i] = qd[d0 + i] + h * vdot[i];
    if (out->vdot) out->vdot[d0 + i] = vdot[i];
  }
  if (out->dynamics_factor) {
    /* LDL^T storage: below the diagonal L_ik d_k = Lc_ik Lc_kk, d_k = Lc_kk^2 */
    double* Lg = out->dynamics_factor + (size_t)e * n * n;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k <= i; ++k) Lg[(size_t)i * n + k] = L[(size_t)i * n + k] * L[(size_t)k * n + k];
  }
  if (out->body_q)
    for (int b = 0; b < B; ++b)
      for (int k = 0; k < 7; ++k) out->body_q[7 * (size_t)(b0g + b) + k] = pose[7 * b + k];

  /* contact rows of this world in flat order (sim/contact_jacobian.py:404-562, 153-251) */
  const int total = world_total[e];
  const int cnt = total < C ? total : C;
  if (out->contact_count) out->contact_count[e] = total;
  for (int c = 0; c < cnt; ++c) {
    const int src = slot_src[(size_t)e * C + c];
    const int sh0 = in->contact_shape0[src], sh1 = in->contact_shape1[src];
    const int gb0 = (sh0 >= 0 && sh0 < m->num_shapes) ? m->shape_body[sh0] : -1;
    const int gb1 = (sh1 >= 0 && sh1 < m->num_shapes) ? m->shape_body[sh1] : -1;
    const int lb0 = gb0 >= 0 ? gb0 - b0g : -1, lb1 = gb1 >= 0 ? gb1 - b0g : -1;
    v3_t x0 = vload(in->contact_point0 + 3 * (size_t)src), x1 = vload(in->contact_point1 + 3 * (size_t)src);
    v3_t p0 = v3(0, 0, 0), p1 = v3(0, 0, 0);
    if (lb0 >= 0) {
      p0 = vload(pose + 7 * lb0);
      x0 = vadd(p0, qrot(qnorm(*(const q4_t*)(pose + 7 * lb0 + 3)), x0));
    }
    if (lb1 >= 0) {
      p1 = vload(pose + 7 * lb1);
      x1 = vadd(p1, qrot(qnorm(*(const q4_t*)(pose + 7 * lb1 + 3)), x1));
    }
    v3_t nrm = vload(in->contact_normal + 3 * (size_t)src);
    const double nn = sqrt(dot3(nrm, nrm));
    if (nn > 0.0) nrm = vscale(1.0 / nn, nrm);
    double F[9];
    contact_frame(nrm, F);
    const double k0 = mat_k(m, o, sh0), k1 = mat_k(m, o, sh1), den = k0 + k1;
    const double w0 = den != 0.0 ? k0 / den : 0.5, w1 = den != 0.0 ? k1 / den : 0.5;
    const v3_t pC = vadd(vscale(w0, x0), vscale(w1, x1));
    const size_t ci = (size_t)e * C + c;
    const double m0 = in->contact_margin0 ? in->contact_margin0[src] : 0.0;
    const double m1 = in->contact_margin1 ? in->contact_margin1[src] : 0.0;
    out->phi0[ci] = dot3(vsub(x1, x0), nrm) - m0 - m1;
    const double mu0 = mat_mu(m, o, sh0), mu1 = mat_mu(m, o, sh1), mden = mu0 + mu1;
    out->mu[ci] = mden <= 1.0e-12 ? 0.0 : 2.0 * mu0 * mu1 / mden;
    out->stiffness[ci] = !isfinite(k0) ? k1 : (!isfinite(k1) ? k0 : (den <= 1.0e-12 ? fmax(k0, k1) : k0 * k1 / den));
    out->tau_d[ci] = mat_tau(m, o, sh0) + mat_tau(m, o, sh1);
    out->body0[ci] = gb0;
    out->body1[ci] = gb1;
    if (out->point) vstore(out->point + 3 * ci, pC);
    if (out->frame) memcpy(out->frame + 9 * ci, F, sizeof(F));
    const int mid = o->contact_point_mode == SAPB_POINT_MIDPOINT;
    const v3_t xj0 = mid ? pC : x0, xj1 = mid ? pC : x1;
    double* Jrow = out->jacobian + ci * 3 * n;
    double wq[6] = {0, 0, 0, 0, 0, 0}, vc[3] = {0, 0, 0};
    for (int col = 0; col < n; ++col) {
      v3_t rel = v3(0, 0, 0);
      if (lb1 >= 0) {
        const double* J = Jb + (size_t)lb1 * 6 * n + col;
        const v3_t w = v3(J[0], J[n], J[2 * n]), v = v3(J[3 * n], J[4 * n], J[5 * n]);
        rel = vadd(rel, vadd(v, vcross(w, vsub(xj1, p1))));
      }
      if (lb0 >= 0) {
        const double* J = Jb + (size_t)lb0 * 6 * n + col;
        const v3_t w = v3(J[0], J[n], J[2 * n]), v = v3(J[3 * n], J[4 * n], J[5 * n]);
        rel = vsub(rel, vadd(v, vcross(w, vsub(xj0, p0))));
      }
      double r3[3];
      for (int r = 0; r < 3; ++r) {
        r3[r] = F[3 * r] * rel.x + F[3 * r + 1] * rel.y + F[3 * r + 2] * rel.z;
        Jrow[(size_t)r * n + col] = r3[r];
      }
      const double vs = out->v_star[d0 + col];
      for (int r = 0; r < 3; ++r) vc[r] += r3[r] * vs;
      double aii = A[(size_t)col * n + col];
      if (aii < 1.0e-12) aii = 1.0e-12;
      const double inv = 1.0 / aii;
      wq[0] += inv * r3[0] * r3[0];
      wq[1] += inv * r3[0] * r3[1];
      wq[2] += inv * r3[0] * r3[2];
      wq[3] += inv * r3[1] * r3[1];
      wq[4] += inv * r3[1] * r3[2];
      wq[5] += inv * r3[2] * r3[2];
    }
    if (out->vc_star)
      for (int r = 0; r < 3; ++r) out->vc_star[3 * ci + r] = vc[r];
    double wv = 0.0;
    if (o->contact_weight_mode == SAPB_WEIGHT_DIAG_DELASSUS) {
      wv = sqrt(wq[0] * wq[0] + wq[3] * wq[3] + wq[5] * wq[5] + 2.0 * (wq[1] * wq[1] + wq[2] * wq[2] + wq[4] * wq[4])) /
           3.0;
    } else {
      /* body-inertia weights use the witnesses, whatever the point mode */
      double wsum = 0.0;
      const int lbs[2] = {lb0, lb1};
      const double* xl[2] = {in->contact_point0 + 3 * (size_t)src, in->contact_point1 + 3 * (size_t)src};
      for (int side = 0; side < 2; ++side) {
        const int lb = lbs[side];
        if (lb < 0) continue;
        const double mass = m->body_mass[b0g + lb];
        if (mass <= 1.0e-12) continue;
        const q4_t qq = qnorm(*(const q4_t*)(pose + 7 * lb + 3));
        const v3_t pb = vload(pose + 7 * lb);
        const v3_t xw = vadd(pb, qrot(qq, vload(xl[side])));
        const v3_t com = vadd(pb, qrot(qq, vload(m->body_com + 3 * (size_t)(b0g + lb))));
        const v3_t r = vsub(xw, com);
        const double* Ic = m->body_inertia + 9 * (size_t)(b0g + lb);
        const double ix = fmax(Ic[0], 1.0e-12), iy = fmax(Ic[4], 1.0e-12), iz = fmax(Ic[8], 1.0e-12);
        for (int d = 0; d < 3; ++d) {
          const v3_t cb = qrot(qconj(qq), vcross(r, vload(F + 3 * d)));
          wsum += 1.0 / mass + cb.x * cb.x / ix + cb.y * cb.y / iy + cb.z * cb.z / iz;
        }
      }
      wv = wsum / 3.0;
    }
    out->w_eff[ci] = wv < 1.0e-12 ? 1.0e-12 : wv;
  }
  free(pose);
  free(V);
  free(Ab);
  free(S);
  free(I6);
  free(fbody);
  free(ft);
  free(tau);
  free(Jb);
  free(A);
  free(L);
  free(vdot);
}

int32_t sapo_free_motion_contacts(const sapb_model_desc* m, const sapb_step_inputs* in, const sapb_prepare_options* o,
                                  const sapb_prepare_outputs* out, int32_t num_threads) {
  if (!m || !in || !o || !out || !out->v_star || !out->dynamics_matrix) return SAPB_ERR_INVALID_ARGUMENT;
  const int W = m->num_worlds, B = m->bodies_per_world, C = o->max_contacts;
  int32_t* total = (int32_t*)calloc((size_t)(W > 0 ? W : 1), sizeof(int32_t));
  int32_t* src = (int32_t*)calloc((size_t)(W > 0 ? W : 1) * (C > 0 ? C : 1), sizeof(int32_t));
  int32_t truncated = 0;
  /* scatter in flat order (_contact_env_from_shapes, sim/sap_helpers.py:439-464) */
  int live = in->contact_count ? in->contact_count[0] : 0;
  if (live > in->contact_capacity) live = in->contact_capacity;
  const int nb = B * W;
  for (int t = 0; t < live; ++t) {
    const int sh0 = in->contact_shape0[t], sh1 = in->contact_shape1[t];
    const int b0 = (sh0 >= 0 && sh0 < m->num_shapes) ? m->shape_body[sh0] : -1;
    const int b1 = (sh1 >= 0 && sh1 < m->num_shapes) ? m->shape_body[sh1] : -1;
    int env = -1;
    if (b0 >= 0 && b0 < nb) env = b0 / B;
    else if (b1 >= 0 && b1 < nb) env = b1 / B;
    if (env < 0) continue;
    if (b0 >= 0 && (b0 >= nb || b0 / B != env)) continue;
    if (b1 >= 0 && (b1 >= nb || b1 / B != env)) continue;
    const int slot = total[env]++;
    if (slot < C) src[(size_t)env * C + slot] = t;
    else ++truncated;
  }
  if (out->truncated_count) out->truncated_count[0] = truncated;
  if (num_threads > 0) omp_set_num_threads(num_threads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < W; ++e) world_step(m, in, o, out, src, total, e);
  free(total);
  free(src);
  return SAPB_OK;
}

int32_t sapo_integrate_positions(const sapb_model_desc* m, const double* q_in, const double* v_prev,
                                 const double* v_new, const double* dt, int32_t mode, double* q_out) {
  /* sim/solver_sap.py:144-733: sap_euler q' = q + dt 0.5 [0, w] q, midpoint exp map;
   * coordinates of fixed joints are copied */
  const int J = m->joints_per_world * m->num_worlds;
  if (q_out != q_in) memcpy(q_out, q_in, sizeof(double) * (size_t)m->coords_per_world * m->num_worlds);
  for (int j = 0; j < J; ++j) {
    const int jt = m->joint_type[j], qs = m->joint_q_start[j], ds = m->joint_qd_start[j];
    const double h = dt[j / m->joints_per_world];
    const int midp = mode == SAPB_INTEGRATE_MIDPOINT;
#define VEL(k) (midp ? 0.5 * (v_prev[(k)] + v_new[(k)]) : v_new[(k)])
    if (jt == SAPB_JOINT_PRISMATIC || jt == SAPB_JOINT_REVOLUTE) {
      q_out[qs] = q_in[qs] + h * VEL(ds);
    } else if (jt == SAPB_JOINT_BALL || jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
      const int off = jt == SAPB_JOINT_BALL ? 0 : 3;
      if (off == 3)
        for (int k = 0; k < 3; ++k) q_out[qs + k] = q_in[qs + k] + h * VEL(ds + 3 + k);
      q4_t qq = {q_in[qs + off], q_in[qs + off + 1], q_in[qs + off + 2], q_in[qs + off + 3]};
      const v3_t w = v3(VEL(ds), VEL(ds + 1), VEL(ds + 2));
      q4_t qn = qq;
      if (!midp) {
        const double hd = 0.5 * h;
        q4_t t = {qq.x + hd * (qq.w * w.x + w.y * qq.z - w.z * qq.y), qq.y + hd * (qq.w * w.y + w.z * qq.x - w.x * qq.z),
                  qq.z + hd * (qq.w * w.z + w.x * qq.y - w.y * qq.x), qq.w - hd * (w.x * qq.x + w.y * qq.y + w.z * qq.z)};
        qn = qnorm(t);
      } else {
        const double wn = sqrt(dot3(w, w)), ang = wn * h;
        if (ang > 1.0e-12) qn = qnorm(qmul(qaxis(vscale(1.0 / wn, w), ang), qq));
      }
      q_out[qs + off] = qn.x;
      q_out[qs + off + 1] = qn.y;
      q_out[qs + off + 2] = qn.z;
      q_out[qs + off + 3] = qn.w;
    } else if (jt != SAPB_JOINT_FIXED) {
      const int dim = m->joint_dof_dim[2 * j] + m->joint_dof_dim[2 * j + 1];
      for (int k = 0; k < dim; ++k) q_out[qs + k] = q_in[qs + k] + h * VEL(ds + k);
    }
#undef VEL
  }
  return SAPB_OK;
}
