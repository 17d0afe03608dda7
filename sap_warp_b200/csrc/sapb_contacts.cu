// sapb_contacts.cu -- contact generation for primitive shapes (planes,
// spheres, boxes) into the flat contact buffer the step reads.
//
// The reference generates contacts with its collision pipeline (broad phase,
// primitive / GJK-MPR narrow phase) and writes each one with
// sap_write_contact (sim/collision/pipeline.py:52-118): shape pair (a, b),
// witness points in the body frames of their shapes (world frame for static
// shapes), the unit normal from a to b, and margins = effective radius +
// shape margin, so that the step's phi0 = (x_b - x_a) . n - m_a - m_b is the
// signed surface distance.  This file covers the primitive pairs of the
// synthetic scenes with closed-form tests:
//   plane-sphere, plane-box (the deepest four corners), sphere-sphere, sphere-box (closest
//   point), box-box (corners of each box against the faces of the other,
//   and, when a separating-axis test over the 15 axes finds an edge-edge
//   axis the least penetrating, one contact between the two crossing edges,
//   as sap_collide_box_box does for edges, sim/collision/primitive.py:692-1148).
// Spheres keep their centre as the witness point with the radius in the
// margin (the reference's radius_eff); boxes and planes have zero radius.
// A contact is emitted when its signed distance is below the gap.
//
// Output order is deterministic: a count pass per candidate pair, an
// exclusive scan of the counts, and a write pass at the scanned offsets
// (pairs in world order, then by shape index; contacts of a pair in a fixed
// order), so the flat buffer -- and the per-world slot order the step derives
// from it -- is the same on every run.
#include <cuda_runtime.h>

#include <cstdint>

#include "sapb_internal.h"
#include "sapb_spatial.cuh"

namespace sapb {

namespace {

constexpr int kScanBlock = 1024;

struct GenParams {
  sapb_collision_shapes s;
  const double* body_q;
  int32_t num_worlds;
  int64_t pairs_per_world;
  int64_t num_pairs;
};

__device__ __forceinline__ Xf xf_mul_n(Xf a, Xf b) { return Xf{a.p + qrot(a.q, b.p), qmul(a.q, b.q)}; }
__device__ __forceinline__ V3 xf_point(Xf a, V3 p) { return a.p + qrot(a.q, p); }
__device__ __forceinline__ V3 xf_inv_point(Xf a, V3 p) { return qrot(qconj(a.q), p - a.p); }

// world pose of a shape: body pose o shape frame (static shapes: the frame)
__device__ Xf shape_world(const GenParams& P, int sh) {
  const Xf X_bs = xf_load(P.s.shape_X_bs + 7 * (size_t)sh);
  const int b = P.s.shape_body[sh];
  if (b < 0) return X_bs;
  return xf_mul_n(xf_load(P.body_q + 7 * (size_t)b), X_bs);
}

__device__ V3 body_local(const GenParams& P, int sh, V3 pw) {
  const int b = P.s.shape_body[sh];
  if (b < 0) return pw;
  return xf_inv_point(xf_load(P.body_q + 7 * (size_t)b), pw);
}

// The pair k of a world: first each local shape against each global shape,
// then the local pairs (i < j).  Shapes: Sw local per world, then G global.
__device__ void decode_pair(const GenParams& P, int64_t k, int w, int* a, int* b) {
  const int Sw = P.s.shapes_per_world, G = P.s.num_global_shapes;
  const int base = w * Sw, gbase = P.num_worlds * Sw;
  if (k < (int64_t)Sw * G) {
    *a = gbase + (int)(k % G);  // the global shape (static plane) first: normal from it to the local shape
    *b = base + (int)(k / G);
    return;
  }
  int64_t q = k - (int64_t)Sw * G;
  // row-major upper triangle: i < j
  int i = 0;
  int64_t row = Sw - 1;
  while (q >= row && row > 0) {
    q -= row;
    ++i;
    --row;
  }
  *a = base + i;
  *b = base + i + 1 + (int)q;
}

struct Emit {
  // count mode when out == nullptr
  const GenParams* P;
  int64_t at;
  int n;
  const sapb_contact_outputs* out;
  __device__ void operator()(int sa, int sb, V3 xa_w, V3 xb_w, V3 nrm, double ma, double mb) {
    if (out) {
      const int64_t i = at + n;
      if (i < out->capacity) {
        out->shape0[i] = sa;
        out->shape1[i] = sb;
        store3(out->point0 + 3 * i, body_local(*P, sa, xa_w));
        store3(out->point1 + 3 * i, body_local(*P, sb, xb_w));
        store3(out->normal + 3 * i, nrm);
        out->margin0[i] = ma;
        out->margin1[i] = mb;
      }
    }
    ++n;
  }
};

__device__ __forceinline__ V3 box_corner(V3 h, int c) {
  return v3((c & 1) ? h.x : -h.x, (c & 2) ? h.y : -h.y, (c & 4) ? h.z : -h.z);
}

__device__ void box_corners_vs_box(const GenParams& P, int sa_box, int sb_vert, Xf Xa, V3 ha, Xf Xb, V3 hb,
                                   double gap, double ma, double mb, Emit& emit) {
  // corners of box sb_vert against the faces of box sa_box; normal from sa_box to sb_vert
  for (int c = 0; c < 8; ++c) {
    const V3 vw = xf_point(Xb, box_corner(hb, c));
    const V3 p = xf_inv_point(Xa, vw);
    const double ex = fabs(p.x) - ha.x, ey = fabs(p.y) - ha.y, ez = fabs(p.z) - ha.z;
    if (ex > gap || ey > gap || ez > gap) continue;
    // the face of least penetration (largest e)
    int k = 0;
    double e = ex;
    if (ey > e) {
      k = 1;
      e = ey;
    }
    if (ez > e) {
      k = 2;
      e = ez;
    }
    const double s = k == 0 ? (p.x >= 0 ? 1.0 : -1.0) : k == 1 ? (p.y >= 0 ? 1.0 : -1.0) : (p.z >= 0 ? 1.0 : -1.0);
    V3 nl = v3(k == 0 ? s : 0.0, k == 1 ? s : 0.0, k == 2 ? s : 0.0);
    V3 face = p;
    if (k == 0) face.x = s * ha.x;
    if (k == 1) face.y = s * ha.y;
    if (k == 2) face.z = s * ha.z;
    emit(sa_box, sb_vert, xf_point(Xa, face), vw, qrot(Xa.q, nl), ma, mb);
  }
}

// Edge-edge contact of two boxes (normal from a to b): the separating-axis
// test over the 3 + 3 face axes and the 9 edge-pair axes; when the best
// (least penetrating) edge axis beats every face axis by a relative 1e-6 and
// lies within the gap, the two edges supporting it (A's farthest along the
// axis, B's farthest against it) give one contact at their closest points,
// provided those lie inside both edges (the edges cross; otherwise a corner
// is involved and the vertex-face tests cover it).
__device__ void box_edge_contact(int a, int b, Xf Xa, V3 ha, Xf Xb, V3 hb, double gap, double ma, double mb,
                                 Emit& emit) {
  const V3 A[3] = {qrot(Xa.q, v3(1, 0, 0)), qrot(Xa.q, v3(0, 1, 0)), qrot(Xa.q, v3(0, 0, 1))};
  const V3 B[3] = {qrot(Xb.q, v3(1, 0, 0)), qrot(Xb.q, v3(0, 1, 0)), qrot(Xb.q, v3(0, 0, 1))};
  const double hA[3] = {ha.x, ha.y, ha.z}, hB[3] = {hb.x, hb.y, hb.z};
  const V3 d = Xb.p - Xa.p;
  auto radius = [&](const V3* E, const double* h, V3 L) {
    return h[0] * fabs(dot(E[0], L)) + h[1] * fabs(dot(E[1], L)) + h[2] * fabs(dot(E[2], L));
  };
  double best_face = -1.0e300;
  for (int k = 0; k < 3; ++k) {
    const double sa = fabs(dot(d, A[k])) - (hA[k] + radius(B, hB, A[k]));
    const double sb = fabs(dot(d, B[k])) - (radius(A, hA, B[k]) + hB[k]);
    best_face = fmax(best_face, fmax(sa, sb));
  }
  // separated along a face axis by the gap or more: no edge axis can be both
  // better and within the gap
  if (!(best_face < gap)) return;
  double best_edge = -1.0e300;
  int bi = -1, bj = -1;
  V3 bL = v3(0, 0, 0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      V3 L = cross(A[i], B[j]);
      const double len = sqrt(dot(L, L));
      if (len < 1.0e-6) continue;  // parallel edges: the face axes decide
      L = (1.0 / len) * L;
      if (dot(d, L) < 0.0) L = -L;
      const double sep = dot(d, L) - radius(A, hA, L) - radius(B, hB, L);
      if (sep > best_edge) {
        best_edge = sep;
        bi = i;
        bj = j;
        bL = L;
      }
    }
  const double scale = fmax(fmax(fmax(hA[0], hA[1]), fmax(hA[2], hB[0])), fmax(hB[1], hB[2]));
  if (bi < 0 || !(best_edge > best_face + 1.0e-6 * scale) || !(best_edge < gap)) return;
  V3 cA = Xa.p, cB = Xb.p;
  for (int m = 0; m < 3; ++m) {
    if (m != bi) cA = cA + (dot(A[m], bL) >= 0.0 ? hA[m] : -hA[m]) * A[m];
    if (m != bj) cB = cB - (dot(B[m], bL) >= 0.0 ? hB[m] : -hB[m]) * B[m];
  }
  const V3 u = A[bi], v = B[bj], w = cA - cB;
  const double uv = dot(u, v), uw = dot(u, w), vw = dot(v, w);
  const double den = 1.0 - uv * uv;
  if (den < 1.0e-12) return;
  const double s = (uv * vw - uw) / den, t = (vw - uv * uw) / den;
  if (fabs(s) > hA[bi] || fabs(t) > hB[bj]) return;
  emit(a, b, cA + s * u, cB + t * v, bL, ma, mb);
}

// sap_test_group_pair (sim/collision/broad_phase_common.py:133-150)
__device__ __forceinline__ bool groups_meet(int ga, int gb) {
  if (ga == 0 || gb == 0) return false;
  if (ga > 0) return ga == gb || gb < 0;
  return ga != gb;
}

__device__ void pair_contacts(const GenParams& P, int sa, int sb, Emit& emit) {
  if (P.s.shape_collision_group &&
      !groups_meet(P.s.shape_collision_group[sa], P.s.shape_collision_group[sb]))
    return;
  const int ta = P.s.shape_type[sa], tb = P.s.shape_type[sb];
  const double gap = P.s.gap;
  const double mga = P.s.shape_margin ? P.s.shape_margin[sa] : 0.0;
  const double mgb = P.s.shape_margin ? P.s.shape_margin[sb] : 0.0;
  // order each pair as (plane | sphere | box) by type rank so the cases below
  // see a fixed order; the normal always points from the first to the second
  int a = sa, b = sb, t1 = ta, t2 = tb;
  double m1 = mga, m2 = mgb;
  if (t1 > t2) {
    a = sb;
    b = sa;
    t1 = tb;
    t2 = ta;
    m1 = mgb;
    m2 = mga;
  }
  const Xf Xa = shape_world(P, a), Xb = shape_world(P, b);
  const V3 sa3 = load3(P.s.shape_scale + 3 * (size_t)a), sb3 = load3(P.s.shape_scale + 3 * (size_t)b);
  if (t1 == SAPB_SHAPE_PLANE && t2 == SAPB_SHAPE_PLANE) return;
  if (t1 != SAPB_SHAPE_PLANE) {
    // bounding spheres (a sphere's radius, a box's half diagonal): pairs
    // farther apart than both plus sqrt(3) x (margins + gap) cannot touch
    // (the box tests accept a corner up to that far out on every axis at
    // once); the slack keeps the cut conservative under rounding
    const double ra = t1 == SAPB_SHAPE_SPHERE ? sa3.x : sqrt(dot(sa3, sa3));
    const double rb = t2 == SAPB_SHAPE_SPHERE ? sb3.x : sqrt(dot(sb3, sb3));
    const V3 d = Xb.p - Xa.p;
    const double reach =
        (ra + rb + 1.7320508075688772 * (fabs(m1) + fabs(m2) + fabs(gap))) * (1.0 + 1.0e-12) + 1.0e-12;
    if (dot(d, d) > reach * reach) return;
  }
  if (t1 == SAPB_SHAPE_PLANE) {
    const V3 n = qrot(Xa.q, v3(0, 0, 1));
    if (t2 == SAPB_SHAPE_SPHERE) {
      const double d = dot(Xb.p - Xa.p, n) - sb3.x;
      if (d - m1 - m2 < gap) emit(a, b, Xb.p - dot(Xb.p - Xa.p, n) * n, Xb.p, n, m1, sb3.x + m2);
    } else if (t2 == SAPB_SHAPE_BOX) {
      // the corners within the gap, at most four: the deepest ones, kept in
      // slots as sap_collide_plane_box does (sim/collision/primitive.py:354-428)
      double kd[4];
      int kc[4];
      int nk = 0, worst = 0;
      for (int c = 0; c < 8; ++c) {
        const V3 vw = xf_point(Xb, box_corner(sb3, c));
        const double d = dot(vw - Xa.p, n);
        if (!(d - m1 - m2 < gap)) continue;
        if (nk < 4) {
          kd[nk] = d;
          kc[nk] = c;
          if (nk == 0 || d > kd[worst]) worst = nk;
          ++nk;
        } else if (d < kd[worst]) {
          kd[worst] = d;
          kc[worst] = c;
          worst = 0;
          for (int i = 1; i < 4; ++i)
            if (kd[i] > kd[worst]) worst = i;
        }
      }
      for (int i = 0; i < nk; ++i) {
        const V3 vw = xf_point(Xb, box_corner(sb3, kc[i]));
        emit(a, b, vw - kd[i] * n, vw, n, m1, m2);
      }
    }
    return;
  }
  if (t1 == SAPB_SHAPE_SPHERE && t2 == SAPB_SHAPE_SPHERE) {
    const V3 dlt = Xb.p - Xa.p;
    const double dist = sqrt(dot(dlt, dlt));
    if (dist - sa3.x - sb3.x - m1 - m2 >= gap) return;
    const V3 n = dist > 1.0e-12 ? (1.0 / dist) * dlt : v3(0, 0, 1);
    emit(a, b, Xa.p, Xb.p, n, sa3.x + m1, sb3.x + m2);
    return;
  }
  if (t1 == SAPB_SHAPE_SPHERE && t2 == SAPB_SHAPE_BOX) {
    // normal from the box (b) to the sphere (a): emit with the box first
    const V3 c = xf_inv_point(Xb, Xa.p);
    V3 p = v3(fmin(fmax(c.x, -sb3.x), sb3.x), fmin(fmax(c.y, -sb3.y), sb3.y), fmin(fmax(c.z, -sb3.z), sb3.z));
    V3 nl;
    const V3 dl = c - p;
    const double dd = sqrt(dot(dl, dl));
    double d;
    if (dd > 1.0e-12) {
      nl = (1.0 / dd) * dl;
      d = dd;
    } else {  // centre inside: the face of least penetration
      const double ex = fabs(c.x) - sb3.x, ey = fabs(c.y) - sb3.y, ez = fabs(c.z) - sb3.z;
      int k = 0;
      double e = ex;
      if (ey > e) {
        k = 1;
        e = ey;
      }
      if (ez > e) {
        k = 2;
        e = ez;
      }
      const double s = k == 0 ? (c.x >= 0 ? 1.0 : -1.0) : k == 1 ? (c.y >= 0 ? 1.0 : -1.0) : (c.z >= 0 ? 1.0 : -1.0);
      nl = v3(k == 0 ? s : 0.0, k == 1 ? s : 0.0, k == 2 ? s : 0.0);
      if (k == 0) p.x = s * sb3.x;
      if (k == 1) p.y = s * sb3.y;
      if (k == 2) p.z = s * sb3.z;
      d = e;
    }
    if (d - sa3.x - m1 - m2 >= gap) return;
    emit(b, a, xf_point(Xb, p), Xa.p, qrot(Xb.q, nl), m2, sa3.x + m1);
    return;
  }
  if (t1 == SAPB_SHAPE_BOX && t2 == SAPB_SHAPE_BOX) {
    box_corners_vs_box(P, a, b, Xa, sa3, Xb, sb3, gap + m1 + m2, m1, m2, emit);
    box_corners_vs_box(P, b, a, Xb, sb3, Xa, sa3, gap + m1 + m2, m2, m1, emit);
    box_edge_contact(a, b, Xa, sa3, Xb, sb3, gap + m1 + m2, m1, m2, emit);
  }
}

__global__ void count_kernel(const GenParams P, int32_t* counts) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= P.num_pairs) return;
  const int w = (int)(t / P.pairs_per_world);
  int a, b;
  decode_pair(P, t - (int64_t)w * P.pairs_per_world, w, &a, &b);
  Emit e{&P, 0, 0, nullptr};
  pair_contacts(P, a, b, e);
  counts[t] = e.n;
}

// Exclusive scan of counts in blocks of kScanBlock (block sums out), then of
// the block sums by one block, then the offsets added in the write pass.
__global__ void scan_blocks_kernel(const int32_t* in, int64_t n, int64_t* out, int64_t* block_sums) {
  __shared__ int64_t s[kScanBlock];
  const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
  const int64_t v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    const int64_t x = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += x;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == kScanBlock - 1) block_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void scan_sums_kernel(int64_t* block_sums, int64_t nb, int32_t* total_out, int32_t capacity) {
  // one block: thread t sums a run of consecutive block sums, the runs'
  // totals are scanned in shared memory, then each run is rewritten as
  // exclusive offsets (integer sums: the same on every run)
  __shared__ int64_t s[kScanBlock];
  const int t = threadIdx.x;
  const int64_t per = (nb + kScanBlock - 1) / kScanBlock;
  const int64_t b0 = (int64_t)t * per;
  const int64_t b1 = b0 + per < nb ? b0 + per : nb;
  int64_t local = 0;
  for (int64_t b = b0; b < b1; ++b) local += block_sums[b];
  s[t] = local;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    const int64_t x = t >= o ? s[t - o] : 0;
    __syncthreads();
    s[t] += x;
    __syncthreads();
  }
  int64_t acc = s[t] - local;
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = block_sums[b];
    block_sums[b] = acc;
    acc += v;
  }
  // The full number of contacts found, like the reference's writer, whose
  // atomic count keeps growing past the buffer (sim/collision/pipeline.py:
  // 87-90): consumers cap it at the buffer length themselves (the step's
  // scatter does), and a count above the capacity tells the caller that the
  // contacts past it were dropped.  Saturates at INT32_MAX.
  (void)capacity;
  if (t == kScanBlock - 1) *total_out = (int32_t)(s[t] < INT32_MAX ? s[t] : INT32_MAX);
}

__global__ void write_kernel(const GenParams P, const int64_t* offsets, const int64_t* block_offsets,
                             const sapb_contact_outputs out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= P.num_pairs) return;
  const int w = (int)(t / P.pairs_per_world);
  int a, b;
  decode_pair(P, t - (int64_t)w * P.pairs_per_world, w, &a, &b);
  Emit e{&P, offsets[t] + block_offsets[t / kScanBlock], 0, &out};
  pair_contacts(P, a, b, e);
}

GenParams make_params(const sapb_collision_shapes* s, const double* body_q) {
  GenParams P;
  P.s = *s;
  P.body_q = body_q;
  P.num_worlds = s->num_worlds;
  const int64_t Sw = s->shapes_per_world, G = s->num_global_shapes;
  P.pairs_per_world = Sw * G + Sw * (Sw - 1) / 2;
  P.num_pairs = P.pairs_per_world * s->num_worlds;
  return P;
}

}  // namespace

size_t contacts_workspace_bytes(const sapb_collision_shapes* s) {
  const GenParams P = make_params(s, nullptr);
  const int64_t nb = (P.num_pairs + kScanBlock - 1) / kScanBlock;
  return (size_t)P.num_pairs * (sizeof(int32_t) + sizeof(int64_t)) + (size_t)(nb + 1) * sizeof(int64_t) + 256;
}

int32_t contacts_launch(const sapb_collision_shapes* s, const double* body_q, const sapb_contact_outputs* out,
                        void* workspace, cudaStream_t stream) {
  const GenParams P = make_params(s, body_q);
  if (P.num_pairs == 0) {
    const cudaError_t err = cudaMemsetAsync(out->count, 0, sizeof(int32_t), stream);
    return err == cudaSuccess ? SAPB_OK : SAPB_ERR_CUDA;
  }
  char* ws = static_cast<char*>(workspace);
  int32_t* counts = reinterpret_cast<int32_t*>(ws);
  size_t off = ((size_t)P.num_pairs * sizeof(int32_t) + 15) / 16 * 16;
  int64_t* offsets = reinterpret_cast<int64_t*>(ws + off);
  off += (size_t)P.num_pairs * sizeof(int64_t);
  int64_t* block_sums = reinterpret_cast<int64_t*>(ws + off);
  const int64_t nb = (P.num_pairs + kScanBlock - 1) / kScanBlock;
  const int threads = 128;
  const unsigned blocks = (unsigned)((P.num_pairs + threads - 1) / threads);
  count_kernel<<<blocks, threads, 0, stream>>>(P, counts);
  scan_blocks_kernel<<<(unsigned)nb, kScanBlock, 0, stream>>>(counts, P.num_pairs, offsets, block_sums);
  scan_sums_kernel<<<1, kScanBlock, 0, stream>>>(block_sums, nb, out->count, out->capacity);
  write_kernel<<<blocks, threads, 0, stream>>>(P, offsets, block_sums, *out);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error("contact generation: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

}  // namespace sapb
