/*
 * CPU oracle for the atom3d_b200 parity tests.
 *
 * TEST INFRASTRUCTURE ONLY: the tests, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use this library as the checker.  The product
 * (package atom3d_b200) never links or calls it.
 *
 * Built with -ffp-contract=off so every float expression rounds operation by
 * operation (no FMA contraction) — the GPU SAT uses explicit round-to-nearest
 * intrinsics for the same reason, which makes SAT results bit-comparable.
 *
 * Contents (reference file:line restated):
 *   orc_udf_exact_f64      FP64 brute force closest point (Ericson regions);
 *                          the distance oracle, independent of the reference.
 *   orc_tri_dist_f64       FP64 distance of point i to triangle fid[i].
 *   orc_ref_udf_bruteforce FP32 Triangle::distance_sq / closest_point /
 *                          barycentric (atom3d/kernels/bvh_kernels.cu:101-222)
 *                          over all faces in order, first minimum wins.
 *   orc_ref_bvh_udf        bvh_udf_kernel (:363-463) over a reference
 *                          build_bvh tree (nodes [Nn,9], tris [F,10]).
 *   orc_sat                triangle_aabb_sat (:285-353).
 *   orc_boxes_hit          "some triangle passes SAT" per box (brute force).
 *   orc_ref_bvh_aabb_hit   bvh_aabb_intersect_kernel hit mask (:555-610) over
 *                          a reference tree (node AABB overlap, then SAT).
 *   orc_octree_traverse    OctreeIndexer.octree_traverse
 *                          (atom3d/grid/octree_indexer.py:470-509) with
 *                          orc_boxes_hit as the per-level test.
 *   orc_morton_encode      OctreeIndexer._ijk_to_morton (:162-172).
 *   orc_flood_fill         flood_fill_kernel + host BFS loop
 *                          (atom3d/kernels/flood_fill_kernels.cu:21-175),
 *                          sequential BFS with the same label rules.
 *   orc_clip_pair          sat_clip_polygon_kernel + clip_with_plane
 *                          (atom3d/kernels/cumtv_kernels.cu:209-265,
 *                          :277-460): Sutherland-Hodgman clip of a triangle
 *                          against the box's 6 planes, centroid projected
 *                          onto the triangle, fan area.
 *   orc_aabb_pair_counts / orc_aabb_pairs_fill
 *                          MeshBVH.intersect_aabb modes 1-3
 *                          (atom3d/core/mesh_bvh.py:297-479) by brute force:
 *                          per box, faces in order, SAT then (modes 2-3)
 *                          the clip.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>


/* ---------------- tiny pthread parallel-for (no OpenMP runtime here) ----- */
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

typedef void (*orc_body_fn)(int64_t i, void* ctx);
typedef struct {
  orc_body_fn fn;
  void* ctx;
  int64_t n, chunk;
  atomic_llong next;
} orc_par_t;

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
  if (g_threads > 0) return g_threads;
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

static void* orc_worker(void* arg) {
  orc_par_t* p = (orc_par_t*)arg;
  for (;;) {
    int64_t s = atomic_fetch_add(&p->next, p->chunk);
    if (s >= p->n) break;
    int64_t e = s + p->chunk < p->n ? s + p->chunk : p->n;
    for (int64_t i = s; i < e; ++i) p->fn(i, p->ctx);
  }
  return NULL;
}

static void par_for(int64_t n, int64_t chunk, orc_body_fn fn, void* ctx) {
  int nt = orc_get_threads();
  if (nt > 64) nt = 64;
  orc_par_t p;
  p.fn = fn; p.ctx = ctx; p.n = n; p.chunk = chunk > 0 ? chunk : 1;
  atomic_init(&p.next, 0);
  if (nt <= 1 || n <= p.chunk) { orc_worker(&p); return; }
  pthread_t th[64];
  for (int t = 0; t < nt; ++t) pthread_create(&th[t], NULL, orc_worker, &p);
  for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
}

typedef struct { double x, y, z; } d3;
typedef struct { float x, y, z; } f3;

static inline d3 dsub(d3 a, d3 b) { d3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline d3 dadd(d3 a, d3 b) { d3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline d3 dscl(d3 a, double s) { d3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static inline d3 ldv(const float* V, int64_t i) { d3 r = {V[3 * i], V[3 * i + 1], V[3 * i + 2]}; return r; }

/* Ericson, Real-Time Collision Detection, 5.1.5: closest point on triangle. */
static d3 closest_pt_tri(d3 p, d3 a, d3 b, d3 c) {
  d3 ab = dsub(b, a), ac = dsub(c, a), ap = dsub(p, a);
  double d1 = ddot(ab, ap), d2 = ddot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return a;
  d3 bp = dsub(p, b);
  double d3_ = ddot(ab, bp), d4 = ddot(ac, bp);
  if (d3_ >= 0 && d4 <= d3_) return b;
  double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0 && d1 >= 0 && d3_ <= 0) {
    double v = d1 / (d1 - d3_);
    return dadd(a, dscl(ab, v));
  }
  d3 cp = dsub(p, c);
  double d5 = ddot(ab, cp), d6 = ddot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return c;
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    double w = d2 / (d2 - d6);
    return dadd(a, dscl(ac, w));
  }
  double va = d3_ * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3_) >= 0 && (d5 - d6) >= 0) {
    double w = (d4 - d3_) / ((d4 - d3_) + (d5 - d6));
    return dadd(b, dscl(dsub(c, b), w));
  }
  double denom = 1.0 / (va + vb + vc);
  double v = vb * denom, w = vc * denom;
  return dadd(a, dadd(dscl(ab, v), dscl(ac, w)));
}

static inline double tri_dist2_f64(d3 p, const float* V, const int32_t* F, int64_t f, d3* cp_out) {
  d3 a = ldv(V, F[3 * f]), b = ldv(V, F[3 * f + 1]), c = ldv(V, F[3 * f + 2]);
  d3 q = closest_pt_tri(p, a, b, c);
  d3 d = dsub(p, q);
  if (cp_out) *cp_out = q;
  return ddot(d, d);
}

typedef struct { const float* V; const int32_t* F; int64_t nf; const float* P; double* dist; int32_t* fid; double* cp; } udf64_ctx;
static void udf64_body(int64_t i, void* c_) {
  udf64_ctx* c = (udf64_ctx*)c_;
  const float* V = c->V; const int32_t* F = c->F; int64_t nf = c->nf; const float* P = c->P;
  double* dist = c->dist; int32_t* fid = c->fid; double* cp = c->cp;
  {
    d3 p = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    double best = INFINITY;
    int64_t bf = -1;
    d3 bc = p;
    for (int64_t f = 0; f < nf; ++f) {
      d3 q;
      double d2 = tri_dist2_f64(p, V, F, f, &q);
      if (d2 < best) { best = d2; bf = f; bc = q; }
    }
    dist[i] = sqrt(best);
    fid[i] = (int32_t)bf;
    if (cp) { cp[3 * i] = bc.x; cp[3 * i + 1] = bc.y; cp[3 * i + 2] = bc.z; }
  }
}
void orc_udf_exact_f64(const float* V, const int32_t* F, int64_t nf, const float* P, int64_t np, double* dist,
                       int32_t* fid, double* cp) {
  udf64_ctx c = {V, F, nf, P, dist, fid, cp};
  par_for(np, 16, udf64_body, &c);
}

void orc_tri_dist_f64(const float* V, const int32_t* F, const float* P, const int32_t* fid, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    d3 p = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    out[i] = fid[i] < 0 ? INFINITY : sqrt(tri_dist2_f64(p, V, F, fid[i], NULL));
  }
}

/* ---------------- FP32 restatement of the reference triangle maths ------ */
static inline f3 fsub(f3 a, f3 b) { f3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline f3 fadd(f3 a, f3 b) { f3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline f3 fscl(f3 a, float s) { f3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline float fdot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 fcross(f3 a, f3 b) {
  f3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}
static inline float fclamp01(float v) { return fmaxf(0.0f, fminf(1.0f, v)); }
static inline float fsignp(float x) { return x >= 0.0f ? 1.0f : -1.0f; }

static float ref_dist_sq(f3 p, f3 a, f3 b, f3 c) {
  f3 v21 = fsub(b, a), p1 = fsub(p, a), v32 = fsub(c, b), p2 = fsub(p, b), v13 = fsub(a, c), p3 = fsub(p, c);
  f3 nor = fcross(v21, v13);
  float nsq = fdot(nor, nor);
  int degen = nsq < 1e-12f;
  float st = 0.0f;
  if (!degen)
    st = fsignp(fdot(fcross(v21, nor), p1)) + fsignp(fdot(fcross(v32, nor), p2)) + fsignp(fdot(fcross(v13, nor), p3));
  if (degen || st < 2.0f) {
    f3 vs[3] = {v21, v32, v13}, ps[3] = {p1, p2, p3};
    float best = INFINITY;
    for (int k = 0; k < 3; ++k) {
      float d = fdot(vs[k], ps[k]) / fmaxf(fdot(vs[k], vs[k]), 1e-12f);
      d = fclamp01(d);
      f3 e = fsub(fscl(vs[k], d), ps[k]);
      float v = fdot(e, e);
      best = k == 0 ? v : fminf(best, v);
    }
    return best;
  }
  float d = fdot(nor, p1);
  return d * d / fmaxf(nsq, 1e-12f);
}

static f3 ref_closest(f3 p, f3 a, f3 b, f3 c) {
  f3 v21 = fsub(b, a), p1 = fsub(p, a), v32 = fsub(c, b), p2 = fsub(p, b), v13 = fsub(a, c), p3 = fsub(p, c);
  f3 nor = fcross(v21, v13);
  float nsq = fdot(nor, nor);
  int degen = nsq < 1e-12f;
  float st = 0.0f;
  if (!degen)
    st = fsignp(fdot(fcross(v21, nor), p1)) + fsignp(fdot(fcross(v32, nor), p2)) + fsignp(fdot(fcross(v13, nor), p3));
  if (degen || st < 2.0f) {
    f3 vs[3] = {v21, v32, v13}, ps[3] = {p1, p2, p3}, os[3] = {a, b, c}, cs[3];
    float ds[3];
    for (int k = 0; k < 3; ++k) {
      float d = fclamp01(fdot(vs[k], ps[k]) / fmaxf(fdot(vs[k], vs[k]), 1e-12f));
      cs[k] = fadd(os[k], fscl(vs[k], d));
      f3 e = fsub(cs[k], p);
      ds[k] = fdot(e, e);
    }
    if (ds[0] < ds[1] && ds[0] < ds[2]) return cs[0];
    if (ds[1] < ds[2]) return cs[1];
    return cs[2];
  }
  float d = fdot(nor, p1);
  return fsub(p, fscl(nor, d / fmaxf(nsq, 1e-12f)));
}

static f3 ref_bary(f3 q, f3 a, f3 b, f3 c) {
  f3 v0 = fsub(b, a), v1 = fsub(c, a), v2 = fsub(q, a);
  float d00 = fdot(v0, v0), d01 = fdot(v0, v1), d11 = fdot(v1, v1), d20 = fdot(v2, v0), d21 = fdot(v2, v1);
  float den = d00 * d11 - d01 * d01;
  float v = (d11 * d20 - d01 * d21) / fmaxf(den, 1e-10f);
  float w = (d00 * d21 - d01 * d20) / fmaxf(den, 1e-10f);
  f3 r = {1.0f - v - w, v, w};
  return r;
}

static inline f3 lfv(const float* V, int64_t i) { f3 r = {V[3 * i], V[3 * i + 1], V[3 * i + 2]}; return r; }

static void ref_finish(f3 p, f3 a, f3 b, f3 c, float best, float* dist, float* cp, float* uvw) {
  f3 q = ref_closest(p, a, b, c);
  *dist = sqrtf(best);
  cp[0] = q.x; cp[1] = q.y; cp[2] = q.z;
  f3 bc = ref_bary(q, a, b, c);
  uvw[0] = bc.x; uvw[1] = bc.y; uvw[2] = bc.z;
}

typedef struct { const float* V; const int32_t* F; int64_t nf; const float* P; float* dist; int32_t* fid; float* cp; float* uvw; } rudf_ctx;
static void rudf_body(int64_t i, void* c_) {
  rudf_ctx* c = (rudf_ctx*)c_;
  const float* V = c->V; const int32_t* F = c->F; int64_t nf = c->nf; const float* P = c->P;
  float* dist = c->dist; int32_t* fid = c->fid; float* cp = c->cp; float* uvw = c->uvw;
  {
    f3 p = lfv(P, i);
    float best = 1e30f;
    int64_t bf = -1;
    for (int64_t f = 0; f < nf; ++f) {
      float d = ref_dist_sq(p, lfv(V, F[3 * f]), lfv(V, F[3 * f + 1]), lfv(V, F[3 * f + 2]));
      if (d < best) { best = d; bf = f; }
    }
    fid[i] = (int32_t)bf;
    if (bf >= 0)
      ref_finish(p, lfv(V, F[3 * bf]), lfv(V, F[3 * bf + 1]), lfv(V, F[3 * bf + 2]), best, &dist[i], &cp[3 * i],
                 &uvw[3 * i]);
  }
}
void orc_ref_udf_bruteforce(const float* V, const int32_t* F, int64_t nf, const float* P, int64_t np, float* dist,
                            int32_t* fid, float* cp, float* uvw) {
  rudf_ctx c = {V, F, nf, P, dist, fid, cp, uvw};
  par_for(np, 16, rudf_body, &c);
}

/* reference tree: node = 9 floats (min3, max3, left, right as int bits, pad);
 * leaf: left = -(start+1), right = -(end+1).  tris = 10 floats (a, b, c, id). */
static inline int32_t fbits(float f) { int32_t i; memcpy(&i, &f, 4); return i; }

static float ref_point_aabb(f3 p, const float* n) {
  float dx = fmaxf(fmaxf(n[0] - p.x, 0.0f), p.x - n[3]);
  float dy = fmaxf(fmaxf(n[1] - p.y, 0.0f), p.y - n[4]);
  float dz = fmaxf(fmaxf(n[2] - p.z, 0.0f), p.z - n[5]);
  return dx * dx + dy * dy + dz * dz;
}

typedef struct { const float* nodes; const float* tris; const float* P; float* dist; int32_t* fid; float* cp; float* uvw; } rbvh_ctx;
static void rbvh_body(int64_t qi, void* c_) {
  rbvh_ctx* c = (rbvh_ctx*)c_;
  const float* nodes = c->nodes; const float* tris = c->tris; const float* P = c->P;
  float* dist = c->dist; int32_t* fid = c->fid; float* cp = c->cp; float* uvw = c->uvw;
  {
    f3 p = lfv(P, qi);
    float best = 1e30f;
    int bf = -1, bt = -1;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      int idx = stack[--sp];
      const float* n = nodes + 9 * (int64_t)idx;
      if (ref_point_aabb(p, n) >= best) continue;
      int l = fbits(n[6]), r = fbits(n[7]);
      if (l < 0) {
        int s = -l - 1, e = -r - 1;
        for (int i = s; i < e; ++i) {
          const float* t = tris + 10 * (int64_t)i;
          f3 a = {t[0], t[1], t[2]}, b = {t[3], t[4], t[5]}, c = {t[6], t[7], t[8]};
          float d = ref_dist_sq(p, a, b, c);
          if (d < best) { best = d; bf = fbits(t[9]); bt = i; }
        }
      } else {
        float d1 = ref_point_aabb(p, nodes + 9 * (int64_t)l), d2 = ref_point_aabb(p, nodes + 9 * (int64_t)r);
        if (d1 < d2) {
          if (d2 < best && sp < 128) stack[sp++] = r;
          if (d1 < best && sp < 128) stack[sp++] = l;
        } else {
          if (d1 < best && sp < 128) stack[sp++] = l;
          if (d2 < best && sp < 128) stack[sp++] = r;
        }
      }
    }
    fid[qi] = bf;
    if (bt >= 0) {
      const float* t = tris + 10 * (int64_t)bt;
      f3 a = {t[0], t[1], t[2]}, b = {t[3], t[4], t[5]}, c = {t[6], t[7], t[8]};
      ref_finish(p, a, b, c, best, &dist[qi], &cp[3 * qi], &uvw[3 * qi]);
    } else {
      dist[qi] = sqrtf(best);
      cp[3 * qi] = p.x; cp[3 * qi + 1] = p.y; cp[3 * qi + 2] = p.z;
    }
  }
}
void orc_ref_bvh_udf(const float* nodes, const float* tris, const float* P, int64_t np, float* dist, int32_t* fid,
                     float* cp, float* uvw) {
  rbvh_ctx c = {nodes, tris, P, dist, fid, cp, uvw};
  par_for(np, 16, rbvh_body, &c);
}

/* ---------------- SAT ----------------------------------------------------- */
static inline float dot3r(float ax, float ay, float az, float bx, float by, float bz) {
  return ax * bx + ay * by + az * bz;
}

int orc_sat(const float* t /* 9 */, const float* mn, const float* mx) {
  const float eps = 1e-6f;
  float c[3], h[3], v[3][3];
  for (int a = 0; a < 3; ++a) {
    c[a] = (mn[a] + mx[a]) * 0.5f;
    h[a] = (mx[a] - mn[a]) * 0.5f;
  }
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) v[k][a] = t[3 * k + a] - c[a];
  for (int a = 0; a < 3; ++a) {
    float lo = fminf(fminf(v[0][a], v[1][a]), v[2][a]);
    float hi = fmaxf(fmaxf(v[0][a], v[1][a]), v[2][a]);
    if (lo > h[a] + eps || hi < -h[a] - eps) return 0;
  }
  float e[3][3];
  for (int a = 0; a < 3; ++a) {
    e[0][a] = v[1][a] - v[0][a];
    e[1][a] = v[2][a] - v[1][a];
    e[2][a] = v[0][a] - v[2][a];
  }
  for (int k = 0; k < 3; ++k) {
    for (int ax = 0; ax < 3; ++ax) {
      float a0, a1, a2;
      if (ax == 0) { a0 = 0.0f; a1 = e[k][2]; a2 = -e[k][1]; }
      else if (ax == 1) { a0 = -e[k][2]; a1 = 0.0f; a2 = e[k][0]; }
      else { a0 = e[k][1]; a1 = -e[k][0]; a2 = 0.0f; }
      float p0 = dot3r(v[0][0], v[0][1], v[0][2], a0, a1, a2);
      float p1 = dot3r(v[1][0], v[1][1], v[1][2], a0, a1, a2);
      float p2 = dot3r(v[2][0], v[2][1], v[2][2], a0, a1, a2);
      float lo = fminf(fminf(p0, p1), p2), hi = fmaxf(fmaxf(p0, p1), p2);
      float rad = h[0] * fabsf(a0) + h[1] * fabsf(a1) + h[2] * fabsf(a2) + eps;
      if (lo > rad || hi < -rad) return 0;
    }
  }
  float w[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
  float nx = e[0][1] * w[2] - e[0][2] * w[1];
  float ny = e[0][2] * w[0] - e[0][0] * w[2];
  float nz = e[0][0] * w[1] - e[0][1] * w[0];
  float d = -dot3r(nx, ny, nz, v[0][0], v[0][1], v[0][2]);
  float r = h[0] * fabsf(nx) + h[1] * fabsf(ny) + h[2] * fabsf(nz) + eps;
  if (fabsf(d) > r) return 0;
  return 1;
}

static void gather_tri(const float* V, const int32_t* F, int64_t f, float* t);

/* "Some triangle hits" per box with the stricter rule of the reference's BVH
 * cull applied per triangle: the triangle's own box must overlap the query
 * box exactly (aabb_overlap, bvh_kernels.cu:241-245, :583) before SAT.  The
 * reference applies that cull to node boxes (unions of up to 4 triangle
 * boxes), so its result lies between this and orc_boxes_hit; the tests use
 * it to show that a voxel the product keeps and the reference drops is hit
 * only within sat_eps outside the triangles' own boxes. */
typedef struct { const float* V; const int32_t* F; int64_t nf; const float* bmin; const float* bmax; uint8_t* hit; } bhx_ctx;
static void bhx_body(int64_t i, void* c_) {
  bhx_ctx* c = (bhx_ctx*)c_;
  const float* mn = c->bmin + 3 * i;
  const float* mx = c->bmax + 3 * i;
  uint8_t h = 0;
  for (int64_t f = 0; f < c->nf && !h; ++f) {
    float t[9];
    gather_tri(c->V, c->F, f, t);
    int ov = 1;
    for (int a = 0; a < 3; ++a) {
      const float lo = fminf(fminf(t[a], t[3 + a]), t[6 + a]), hi = fmaxf(fmaxf(t[a], t[3 + a]), t[6 + a]);
      if (lo > mx[a] || hi < mn[a]) ov = 0;
    }
    if (ov && orc_sat(t, mn, mx)) h = 1;
  }
  c->hit[i] = h;
}
void orc_boxes_hit_exact_box(const float* V, const int32_t* F, int64_t nf, const float* bmin, const float* bmax,
                             int64_t n, uint8_t* hit) {
  bhx_ctx c = {V, F, nf, bmin, bmax, hit};
  par_for(n, 1, bhx_body, &c);
}

static void gather_tri(const float* V, const int32_t* F, int64_t f, float* t) {
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) t[3 * k + a] = V[3 * (int64_t)F[3 * f + k] + a];
}

/* triangle boxes grown by a margin for a cheap pre-reject that never
 * rejects a SAT pass (SAT's own box-axis test is stricter) */
static float* tri_boxes(const float* V, const int32_t* F, int64_t nf) {
  float* b = (float*)malloc(sizeof(float) * 6 * (nf > 0 ? nf : 1));
  for (int64_t f = 0; f < nf; ++f) {
    float t[9];
    gather_tri(V, F, f, t);
    for (int a = 0; a < 3; ++a) {
      float lo = fminf(fminf(t[a], t[3 + a]), t[6 + a]), hi = fmaxf(fmaxf(t[a], t[3 + a]), t[6 + a]);
      float g = 1e-5f + 1e-6f * fmaxf(fabsf(lo), fabsf(hi));
      b[6 * f + a] = lo - g;
      b[6 * f + 3 + a] = hi + g;
    }
  }
  return b;
}

static int box_hits(const float* V, const int32_t* F, int64_t nf, const float* tb, const float* mn, const float* mx) {
  for (int64_t f = 0; f < nf; ++f) {
    const float* b = tb + 6 * f;
    if (b[0] > mx[0] || b[3] < mn[0] || b[1] > mx[1] || b[4] < mn[1] || b[2] > mx[2] || b[5] < mn[2]) continue;
    float t[9];
    gather_tri(V, F, f, t);
    if (orc_sat(t, mn, mx)) return 1;
  }
  return 0;
}

typedef struct { const float* V; const int32_t* F; int64_t nf; const float* tb; const float* bmin; const float* bmax; uint8_t* hit; } bh_ctx;
static void bh_body(int64_t i, void* c_) {
  bh_ctx* c = (bh_ctx*)c_;
  c->hit[i] = (uint8_t)box_hits(c->V, c->F, c->nf, c->tb, c->bmin + 3 * i, c->bmax + 3 * i);
}
void orc_boxes_hit(const float* V, const int32_t* F, int64_t nf, const float* bmin, const float* bmax, int64_t n,
                   uint8_t* hit) {
  float* tb = tri_boxes(V, F, nf);
  bh_ctx c = {V, F, nf, tb, bmin, bmax, hit};
  par_for(n, 64, bh_body, &c);
  free(tb);
}

typedef struct { const float* nodes; const float* tris; const float* bmin; const float* bmax; uint8_t* hit; } rah_ctx;
static void rah_body(int64_t q, void* c_) {
  rah_ctx* c = (rah_ctx*)c_;
  const float* nodes = c->nodes; const float* tris = c->tris; const float* bmin = c->bmin; const float* bmax = c->bmax;
  uint8_t* hit = c->hit;
  {
    const float* mn = bmin + 3 * q;
    const float* mx = bmax + 3 * q;
    int any = 0;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      int idx = stack[--sp];
      const float* nd = nodes + 9 * (int64_t)idx;
      int ov = (nd[0] <= mx[0] && nd[3] >= mn[0]) && (nd[1] <= mx[1] && nd[4] >= mn[1]) &&
               (nd[2] <= mx[2] && nd[5] >= mn[2]);
      if (!ov) continue;
      int l = fbits(nd[6]), r = fbits(nd[7]);
      if (l < 0) {
        int s = -l - 1, e = -r - 1;
        for (int i = s; i < e; ++i)
          if (orc_sat(tris + 10 * (int64_t)i, mn, mx)) any = 1;
      } else if (sp < 127) {
        stack[sp++] = r;
        stack[sp++] = l;
      }
    }
    hit[q] = (uint8_t)any;
  }
}
void orc_ref_bvh_aabb_hit(const float* nodes, const float* tris, const float* bmin, const float* bmax, int64_t n,
                          uint8_t* hit) {
  rah_ctx c = {nodes, tris, bmin, bmax, hit};
  par_for(n, 64, rah_body, &c);
}

/* Uniform-grid broadphase over the grown triangle boxes: a triangle is listed
 * in every cell its box overlaps, a query box visits every cell it overlaps
 * (one cell of slack per side), so a triangle whose box overlaps the query's
 * is always met.  The decision per triangle is box_hits' (pre-reject, then
 * SAT), so the result equals the brute-force scan; only the cost changes. */
typedef struct { double lo[3], inv[3]; int g; int64_t* start; int32_t* items; } tgrid_t;

static inline int tgrid_cell(const tgrid_t* G, int a, double x) {
  double t = floor((x - G->lo[a]) * G->inv[a]);
  if (t < 0) t = 0;
  if (t > G->g - 1) t = G->g - 1;
  return (int)t;
}

static void tgrid_build(tgrid_t* G, const float* tb, int64_t nf, const float* lo, const float* ext) {
  int g = (int)(2.0 * cbrt((double)(nf > 1 ? nf : 1)));
  if (g < 4) g = 4;
  if (g > 256) g = 256;
  G->g = g;
  for (int a = 0; a < 3; ++a) {
    G->lo[a] = lo[a];
    G->inv[a] = ext[a] > 0 ? g / (double)ext[a] : 0.0;
  }
  int64_t nc = (int64_t)g * g * g;
  G->start = (int64_t*)calloc((size_t)nc + 1, sizeof(int64_t));
  for (int pass = 0; pass < 2; ++pass) {
    int64_t* fill = NULL;
    if (pass == 1) {
      for (int64_t c = 0; c < nc; ++c) G->start[c + 1] += G->start[c];
      G->items = (int32_t*)malloc(sizeof(int32_t) * (size_t)(G->start[nc] > 0 ? G->start[nc] : 1));
      fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)nc);
      memcpy(fill, G->start, sizeof(int64_t) * (size_t)nc);
    }
    for (int64_t f = 0; f < nf; ++f) {
      const float* b = tb + 6 * f;
      int i0[3], i1[3];
      for (int a = 0; a < 3; ++a) {
        i0[a] = tgrid_cell(G, a, b[a]);
        i1[a] = tgrid_cell(G, a, b[3 + a]);
      }
      for (int x = i0[0]; x <= i1[0]; ++x)
        for (int y = i0[1]; y <= i1[1]; ++y)
          for (int z = i0[2]; z <= i1[2]; ++z) {
            int64_t c = ((int64_t)x * g + y) * g + z;
            if (pass == 0) G->start[c + 1]++;
            else G->items[fill[c]++] = (int32_t)f;
          }
    }
    free(fill);
  }
}

static int tgrid_box_hits(const tgrid_t* G, const float* V, const int32_t* F, const float* tb, const float* mn,
                          const float* mx) {
  int i0[3], i1[3];
  for (int a = 0; a < 3; ++a) {
    i0[a] = tgrid_cell(G, a, mn[a]) - 1;
    i1[a] = tgrid_cell(G, a, mx[a]) + 1;
    if (i0[a] < 0) i0[a] = 0;
    if (i1[a] > G->g - 1) i1[a] = G->g - 1;
  }
  int g = G->g;
  for (int x = i0[0]; x <= i1[0]; ++x)
    for (int y = i0[1]; y <= i1[1]; ++y)
      for (int z = i0[2]; z <= i1[2]; ++z) {
        int64_t c = ((int64_t)x * g + y) * g + z;
        for (int64_t k = G->start[c]; k < G->start[c + 1]; ++k) {
          int64_t f = G->items[k];
          const float* b = tb + 6 * f;
          if (b[0] > mx[0] || b[3] < mn[0] || b[1] > mx[1] || b[4] < mn[1] || b[2] > mx[2] || b[5] < mn[2]) continue;
          float t[9];
          gather_tri(V, F, f, t);
          if (orc_sat(t, mn, mx)) return 1;
        }
      }
  return 0;
}

typedef struct { const float* V; const int32_t* F; const tgrid_t* G; const float* tb; const int64_t* cur; const float* cell; const float* lo; uint8_t* h; } oct_ctx;
static void oct_body(int64_t k, void* c_) {
  oct_ctx* c = (oct_ctx*)c_;
  float mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = (float)c->cur[3 * k + a] * c->cell[a] + c->lo[a];
    mx[a] = mn[a] + c->cell[a];
  }
  c->h[k] = (uint8_t)tgrid_box_hits(c->G, c->V, c->F, c->tb, mn, mx);
}

/* returns K (>= 0), or -(needed) when out_cap is too small */
int64_t orc_octree_traverse(const float* V, const int32_t* F, int64_t nf, const float* lo, const float* cells,
                            int min_level, int max_level, int64_t* out, int64_t out_cap) {
  float* tb = tri_boxes(V, F, nf);
  tgrid_t G;
  tgrid_build(&G, tb, nf, lo, cells); /* cells[0..2] = the level-0 cell = the whole grid */
  int64_t n = (int64_t)1 << (3 * min_level);
  int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * 3 * n);
  int r = 1 << min_level;
  for (int64_t k = 0; k < n; ++k) {
    cur[3 * k] = k / ((int64_t)r * r);
    cur[3 * k + 1] = (k / r) % r;
    cur[3 * k + 2] = k % r;
  }
  int64_t ncur = n;
  for (int level = min_level; level <= max_level; ++level) {
    const float* cell = cells + 3 * level;
    uint8_t* h = (uint8_t*)malloc(ncur > 0 ? ncur : 1);
    oct_ctx oc = {V, F, &G, tb, cur, cell, lo, h};
    par_for(ncur, 64, oct_body, &oc);
    int64_t m = 0;
    for (int64_t k = 0; k < ncur; ++k) m += h[k];
    if (level == max_level) {
      if (m > out_cap) { free(h); free(cur); free(tb); free(G.start); free(G.items); return -m; }
      int64_t o = 0;
      for (int64_t k = 0; k < ncur; ++k)
        if (h[k]) { memcpy(out + 3 * o, cur + 3 * k, 3 * sizeof(int64_t)); ++o; }
      free(h);
      free(cur);
      free(tb);
      free(G.start);
      free(G.items);
      return m;
    }
    int64_t* nxt = (int64_t*)malloc(sizeof(int64_t) * 3 * 8 * (m > 0 ? m : 1));
    int64_t o = 0;
    for (int64_t k = 0; k < ncur; ++k) {
      if (!h[k]) continue;
      for (int c = 0; c < 8; ++c) {
        nxt[3 * o] = 2 * cur[3 * k] + (c & 1);
        nxt[3 * o + 1] = 2 * cur[3 * k + 1] + ((c >> 1) & 1);
        nxt[3 * o + 2] = 2 * cur[3 * k + 2] + ((c >> 2) & 1);
        ++o;
      }
    }
    free(h);
    free(cur);
    cur = nxt;
    ncur = o;
    if (ncur == 0) break;
  }
  free(cur);
  free(tb);
  free(G.start);
  free(G.items);
  return 0;
}

void orc_morton_encode(const int64_t* ijk, int64_t n, int64_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    int64_t x = ijk[3 * i], y = ijk[3 * i + 1], z = ijk[3 * i + 2], m = 0;
    for (int b = 0; b < 21; ++b) {
      m |= ((x >> b) & 1) << (3 * b);
      m |= ((y >> b) & 1) << (3 * b + 1);
      m |= ((z >> b) & 1) << (3 * b + 2);
    }
    out[i] = m;
  }
}

/* occupancy [D,H,W] (uint8), seed (x along W, y along H, z along D),
 * labels: -2 dry, -1 dam, 1 collision, 2 water */
void orc_flood_fill(const uint8_t* occ, int D, int H, int W, int sx, int sy, int sz, int conn, int32_t* mask) {
  const int64_t nvox = (int64_t)D * H * W;
  for (int64_t i = 0; i < nvox; ++i) mask[i] = -2;
  if (sx < 0 || sx >= W || sy < 0 || sy >= H || sz < 0 || sz >= D) return;
  int64_t* q = (int64_t*)malloc(sizeof(int64_t) * (nvox > 0 ? nvox : 1));
  int64_t qh = 0, qt = 0;
  int64_t s = (int64_t)sz * H * W + (int64_t)sy * W + sx;
  mask[s] = 2;
  q[qt++] = s;
  while (qh < qt) {
    int64_t v = q[qh++];
    int z = (int)(v / ((int64_t)H * W)), y = (int)((v % ((int64_t)H * W)) / W), x = (int)(v % W);
    int coll = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          if (!dx && !dy && !dz) continue;
          int dist = abs(dx) + abs(dy) + abs(dz);
          if (conn == 6 && dist > 1) continue;
          if (conn == 18 && dist > 2) continue;
          int nx = x + dx, ny = y + dy, nz = z + dz;
          if (nx < 0 || nx >= W || ny < 0 || ny >= H || nz < 0 || nz >= D) continue;
          int64_t u = (int64_t)nz * H * W + (int64_t)ny * W + nx;
          if (occ[u]) {
            if (mask[u] == -2) mask[u] = -1;
            coll = 1;
          } else if (mask[u] == -2) {
            mask[u] = 2;
            q[qt++] = u;
          }
        }
    if (coll) mask[v] = 1;
  }
  free(q);
}

/* bvh_udf_kernel restated with counters: counts[0] += node AABB distance
 * evaluations (24-B box reads), counts[1] += triangle distance evaluations
 * (36-B triangle reads), summed over all queries.  Used once to fix the
 * per-query algorithmic traversal bytes of the plain method. */
typedef struct { const float* nodes; const float* tris; const float* P; atomic_llong* cnt; } rcnt_ctx;
static void rcnt_body(int64_t qi, void* c_) {
  rcnt_ctx* c = (rcnt_ctx*)c_;
  const float* nodes = c->nodes; const float* tris = c->tris;
  f3 p = lfv(c->P, qi);
  float best = 1e30f;
  long long nn = 0, nt = 0;
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    int idx = stack[--sp];
    const float* n = nodes + 9 * (int64_t)idx;
    ++nn;
    if (ref_point_aabb(p, n) >= best) continue;
    int l = fbits(n[6]), r = fbits(n[7]);
    if (l < 0) {
      int s = -l - 1, e = -r - 1;
      for (int i = s; i < e; ++i) {
        const float* t = tris + 10 * (int64_t)i;
        f3 a = {t[0], t[1], t[2]}, b = {t[3], t[4], t[5]}, cc = {t[6], t[7], t[8]};
        float d = ref_dist_sq(p, a, b, cc);
        ++nt;
        if (d < best) best = d;
      }
    } else {
      float d1 = ref_point_aabb(p, nodes + 9 * (int64_t)l), d2 = ref_point_aabb(p, nodes + 9 * (int64_t)r);
      nn += 2;
      if (d1 < d2) {
        if (d2 < best && sp < 128) stack[sp++] = r;
        if (d1 < best && sp < 128) stack[sp++] = l;
      } else {
        if (d1 < best && sp < 128) stack[sp++] = l;
        if (d2 < best && sp < 128) stack[sp++] = r;
      }
    }
  }
  atomic_fetch_add(&c->cnt[0], nn);
  atomic_fetch_add(&c->cnt[1], nt);
}
void orc_ref_bvh_udf_counts(const float* nodes, const float* tris, const float* P, int64_t np, int64_t* counts) {
  atomic_llong cnt[2];
  atomic_init(&cnt[0], 0);
  atomic_init(&cnt[1], 0);
  rcnt_ctx c = {nodes, tris, P, cnt};
  par_for(np, 16, rcnt_body, &c);
  counts[0] = atomic_load(&cnt[0]);
  counts[1] = atomic_load(&cnt[1]);
}

/* ------------------------------------------------------------------------
 * Rays, brute force over all faces in face order:
 *   Triangle::ray_intersect  (atom3d/kernels/bvh_kernels.cu:185-202)
 *   Triangle::normal         (:89-99), Triangle::barycentric (:205-221)
 *   bvh_ray_intersect_kernel (:469-553): nearest hit, strict "<" (first wins)
 *   bvh_ray_all_hit_kernel   (:935-1022): every hit 0 < t < max_t that is
 *       not grazing (|n.d| >= 1e-4), sign = sign(n.d)
 *   MeshBVH._bary_from_hit   (atom3d/core/mesh_bvh.py:1218-1244)
 *   MeshBVH._sdf_parity / _signed_crossing_count (:850-948), hits of a ray
 *       ordered by t (the reference's float32 sort key keeps that order
 *       only for ray indices below ~8; the intent is t order)
 * ------------------------------------------------------------------------ */
static inline f3 fsub3(f3 a, f3 b) { f3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline f3 fcross3(f3 a, f3 b) {
  f3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}
static inline float fdot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 ldf(const float* V, int64_t i) { f3 r = {V[3 * i], V[3 * i + 1], V[3 * i + 2]}; return r; }

static float ray_tri_f32(f3 a, f3 b, f3 c, f3 ro, f3 rd) {
  const float eps = 1e-8f;
  const double eps_edge = 1.19209290e-7;
  f3 e1 = fsub3(b, a), e2 = fsub3(c, a);
  f3 h = fcross3(rd, e2);
  float det = fdot3(e1, h);
  if (fabsf(det) < eps) return 1e10f;
  float f = 1.0f / det;
  f3 s = fsub3(ro, a);
  double u = (double)f * (double)fdot3(s, h);
  if (u < -eps_edge || u > 1.0 + eps_edge) return 1e10f;
  f3 q = fcross3(s, e1);
  double v = (double)f * (double)fdot3(rd, q);
  if (v < -eps_edge || u + v > 1.0 + eps_edge) return 1e10f;
  float t = f * fdot3(e2, q);
  return (t > eps) ? t : 1e10f;
}

static f3 tri_normal_f32(f3 a, f3 b, f3 c) {
  f3 n = fcross3(fsub3(b, a), fsub3(c, a));
  float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
  if (len > 1e-10f) {
    float inv = 1.0f / len;
    f3 r = {n.x * inv, n.y * inv, n.z * inv};
    return r;
  }
  f3 z = {0.f, 0.f, 1.f};
  return z;
}

typedef struct {
  const float* V; const int32_t* F; int64_t nf; const float* O; const float* D; float max_t;
  uint8_t* hit; float* t; int32_t* fid; float* hp; float* uvw;
} ray_near_ctx;

static void ray_near_body(int64_t i, void* vc) {
  ray_near_ctx* c = (ray_near_ctx*)vc;
  f3 ro = ldf(c->O, i), rd = ldf(c->D, i);
  float mint = c->max_t;
  int32_t best = -1;
  for (int64_t f = 0; f < c->nf; ++f) {
    f3 a = ldf(c->V, c->F[3 * f]), b = ldf(c->V, c->F[3 * f + 1]), cc = ldf(c->V, c->F[3 * f + 2]);
    float t = ray_tri_f32(a, b, cc, ro, rd);
    if (t < mint) { mint = t; best = (int32_t)f; }
  }
  c->hit[i] = best >= 0;
  c->t[i] = mint;
  c->fid[i] = best;
  if (best >= 0) {
    f3 hp = {ro.x + rd.x * mint, ro.y + rd.y * mint, ro.z + rd.z * mint};
    c->hp[3 * i] = hp.x; c->hp[3 * i + 1] = hp.y; c->hp[3 * i + 2] = hp.z;
    f3 a = ldf(c->V, c->F[3 * best]), b = ldf(c->V, c->F[3 * best + 1]), cc = ldf(c->V, c->F[3 * best + 2]);
    f3 e0 = fsub3(b, a), e1 = fsub3(cc, a), vp = fsub3(hp, a);
    float d00 = fdot3(e0, e0), d01 = fdot3(e0, e1), d11 = fdot3(e1, e1), d20 = fdot3(vp, e0), d21 = fdot3(vp, e1);
    float denom = d00 * d11 - d01 * d01 + 1e-12f;
    float bv = (d11 * d20 - d01 * d21) / denom, bw = (d00 * d21 - d01 * d20) / denom;
    c->uvw[3 * i] = 1.0f - bv - bw; c->uvw[3 * i + 1] = bv; c->uvw[3 * i + 2] = bw;
  } else {
    c->hp[3 * i] = c->hp[3 * i + 1] = c->hp[3 * i + 2] = 0.f;
    c->uvw[3 * i] = c->uvw[3 * i + 1] = c->uvw[3 * i + 2] = 0.f;
  }
}

void orc_ray_nearest(const float* V, const int32_t* F, int64_t nf, const float* O, const float* D, int64_t n,
                     float max_t, uint8_t* hit, float* t, int32_t* fid, float* hp, float* uvw) {
  ray_near_ctx c = {V, F, nf, O, D, max_t, hit, t, fid, hp, uvw};
  par_for(n, 16, ray_near_body, &c);
}

/* every non-grazing hit of ray i, in face order; returns the count, writes
 * at most cap entries */
static int64_t ray_all_one(const float* V, const int32_t* F, int64_t nf, f3 ro, f3 rd, float max_t, int64_t cap,
                           float* ts, int32_t* fids, int32_t* signs) {
  int64_t k = 0;
  for (int64_t f = 0; f < nf; ++f) {
    f3 a = ldf(V, F[3 * f]), b = ldf(V, F[3 * f + 1]), cc = ldf(V, F[3 * f + 2]);
    float t = ray_tri_f32(a, b, cc, ro, rd);
    if (t > 0.0f && t < max_t) {
      f3 nn = tri_normal_f32(a, b, cc);
      float ndotd = fdot3(nn, rd);
      if (ndotd > -1e-4f && ndotd < 1e-4f) continue;
      if (k < cap) { ts[k] = t; fids[k] = (int32_t)f; signs[k] = ndotd > 0.0f ? 1 : -1; }
      ++k;
    }
  }
  return k;
}

void orc_ray_all(const float* V, const int32_t* F, int64_t nf, const float* O, const float* D, int64_t n, float max_t,
                 int64_t cap_per_ray, int32_t* counts, float* t, int32_t* fid, int32_t* sign) {
  for (int64_t i = 0; i < n; ++i) {
    int64_t k = ray_all_one(V, F, nf, ldf(O, i), ldf(D, i), max_t, cap_per_ray, t + i * cap_per_ray,
                            fid + i * cap_per_ray, sign + i * cap_per_ray);
    counts[i] = (int32_t)k;
  }
}

typedef struct {
  const float* V; const int32_t* F; int64_t nf; const float* P; const float* dirs; int ndir; float max_t;
  float coalesce; int32_t* votes;
} parity_ctx;

static void parity_body(int64_t i, void* vc) {
  parity_ctx* c = (parity_ctx*)vc;
  enum { CAP = 4096 };
  float ts[CAP];
  int32_t fids[CAP], sg[CAP];
  int32_t votes = 0;
  for (int d = 0; d < c->ndir; ++d) {
    f3 ro = ldf(c->P, i), rd = ldf(c->dirs, d);
    int64_t k = ray_all_one(c->V, c->F, c->nf, ro, rd, c->max_t, CAP, ts, fids, sg);
    if (k > CAP) k = CAP;
    /* stable insertion sort by t */
    for (int64_t a = 1; a < k; ++a) {
      float tv = ts[a]; int32_t sv = sg[a]; int64_t b = a - 1;
      while (b >= 0 && ts[b] > tv) { ts[b + 1] = ts[b]; sg[b + 1] = sg[b]; --b; }
      ts[b + 1] = tv; sg[b + 1] = sv;
    }
    int32_t sc = 0;
    int64_t a = 0;
    while (a < k) {
      int64_t b = a + 1;
      int32_t cnt = 1, sum = sg[a];
      while (b < k && fabsf(ts[b] - ts[b - 1]) < c->coalesce) { ++cnt; sum += sg[b]; ++b; }
      int32_t sgn = sum > 0 ? 1 : (sum < 0 ? -1 : 0);
      int32_t asum = sum < 0 ? -sum : sum;
      sc += (asum == cnt) ? sgn : (asum % 2) * sgn;
      a = b;
    }
    int32_t asc = sc < 0 ? -sc : sc;
    votes += (asc % 2) == 1;
  }
  c->votes[i] = votes;
}

void orc_parity_votes(const float* V, const int32_t* F, int64_t nf, const float* P, int64_t n, const float* dirs,
                      int ndir, float max_t, float coalesce, int32_t* votes) {
  parity_ctx c = {V, F, nf, P, dirs, ndir, max_t, coalesce, votes};
  par_for(n, 4, parity_body, &c);
}


/* ---------------- triangle/box clipping (intersect_aabb modes 2-3) ------ */
#define CLIP_MAXV 8

/* One Sutherland-Hodgman step against the half space n.p - d <= eps.  An
 * emitted vertex past the 8-vertex buffer is dropped (the reference's
 * buffer would overflow there); the count saturates at 8. */
static int clip_plane(float in[CLIP_MAXV][3], int n_in, const float nrm[3], float d, float out[CLIP_MAXV][3],
                      float eps) {
  if (n_in <= 0) return 0;
  float dist[CLIP_MAXV];
  int ins[CLIP_MAXV];
  for (int i = 0; i < n_in; ++i) {
    dist[i] = in[i][0] * nrm[0] + in[i][1] * nrm[1] + in[i][2] * nrm[2] - d;
    ins[i] = dist[i] <= eps;
  }
  int m = 0;
  for (int i = 0; i < n_in; ++i) {
    const int j = (i + 1 == n_in) ? 0 : i + 1;
    const float* P = in[i];
    const float* Q = in[j];
    const float dP = dist[i], dQ = dist[j];
    if (ins[i] && ins[j]) {
      if (m < CLIP_MAXV) { out[m][0] = Q[0]; out[m][1] = Q[1]; out[m][2] = Q[2]; }
      ++m;
    } else if (ins[i] != ins[j]) {
      const float den = dP - dQ;
      if (fabsf(den) > eps) {
        const float t = dP / den;
        if (m < CLIP_MAXV)
          for (int a = 0; a < 3; ++a) out[m][a] = P[a] + t * (Q[a] - P[a]);
        ++m;
      }
      if (ins[j]) {
        if (m < CLIP_MAXV) { out[m][0] = Q[0]; out[m][1] = Q[1]; out[m][2] = Q[2]; }
        ++m;
      }
    }
    if (m >= CLIP_MAXV) return CLIP_MAXV;
  }
  return m;
}

/* Returns 1 when the clipped polygon is non-empty.  verts (24 floats, zero
 * padded), count, centroid and area follow the reference kernel; area stays
 * 0 for a degenerate triangle (its centroid is then vertex a). */
int orc_clip_pair(const float* mn, const float* mx, const float* t, float eps, float* verts, int* count,
                  float* centroid, float* area) {
  float A[CLIP_MAXV][3], B[CLIP_MAXV][3];
  for (int i = 0; i < 3; ++i)
    for (int a = 0; a < 3; ++a) A[i][a] = t[3 * i + a];
  static const float nrm[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  const float dd[6] = {mx[0], -mn[0], mx[1], -mn[1], mx[2], -mn[2]};
  int n = 3;
  for (int k = 0; k < 6; ++k) {
    n = (k & 1) ? clip_plane(B, n, nrm[k], dd[k], A, eps) : clip_plane(A, n, nrm[k], dd[k], B, eps);
    if (!n) {
      *count = 0;
      *area = 0.0f;
      return 0;
    }
  }
  const int cnt = n > CLIP_MAXV ? CLIP_MAXV : n;
  *count = cnt;
  for (int i = 0; i < CLIP_MAXV; ++i)
    for (int a = 0; a < 3; ++a) verts[3 * i + a] = i < cnt ? A[i][a] : 0.0f;
  *area = 0.0f;
  float c[3] = {0.0f, 0.0f, 0.0f};
  for (int i = 0; i < cnt; ++i)
    for (int a = 0; a < 3; ++a) c[a] += A[i][a];
  for (int a = 0; a < 3; ++a) {
    c[a] /= (float)cnt;
    c[a] = fminf(fmaxf(c[a], mn[a]), mx[a]);
  }
  const float ax = t[0], ay = t[1], az = t[2], bx = t[3], by = t[4], bz = t[5], qx = t[6], qy = t[7], qz = t[8];
  const float e1x = bx - ax, e1y = by - ay, e1z = bz - az;
  const float e2x = qx - ax, e2y = qy - ay, e2z = qz - az;
  const float vx = c[0] - ax, vy = c[1] - ay, vz = c[2] - az;
  const float d00 = e1x * e1x + e1y * e1y + e1z * e1z;
  const float d01 = e1x * e2x + e1y * e2y + e1z * e2z;
  const float d11 = e2x * e2x + e2y * e2y + e2z * e2z;
  const float d20 = vx * e1x + vy * e1y + vz * e1z;
  const float d21 = vx * e2x + vy * e2y + vz * e2z;
  const float den = d00 * d11 - d01 * d01;
  if (fabsf(den) < eps * eps) {
    centroid[0] = ax; centroid[1] = ay; centroid[2] = az;
    return 1;
  }
  float v = (d11 * d20 - d01 * d21) / den;
  float w = (d00 * d21 - d01 * d20) / den;
  float u = 1.0f - v - w;
  if (u < 0) u = 0;
  if (v < 0) v = 0;
  if (w < 0) w = 0;
  float nn = u + v + w;
  if (nn <= eps) { u = 1; v = 0; w = 0; nn = 1; }
  u /= nn; v /= nn; w /= nn;
  centroid[0] = u * ax + v * bx + w * qx;
  centroid[1] = u * ay + v * by + w * qy;
  centroid[2] = u * az + v * bz + w * qz;
  float ar = 0.0f;
  for (int i = 0; i < cnt; ++i) {
    const int j = (i + 1) % cnt;
    const float p0 = A[i][0] - c[0], p1 = A[i][1] - c[1], p2 = A[i][2] - c[2];
    const float q0 = A[j][0] - c[0], q1 = A[j][1] - c[1], q2 = A[j][2] - c[2];
    const float cx = p1 * q2 - p2 * q1, cy = p2 * q0 - p0 * q2, cz = p0 * q1 - p1 * q0;
    ar += 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
  }
  *area = ar < eps ? 0.0f : ar;
  return 1;
}

typedef struct {
  const float* V; const int32_t* F; int64_t nf; const float* tb; const float* bmin; const float* bmax;
  int clip; float eps; int64_t* counts; const int64_t* offs;
  int64_t* box_ids; int64_t* face_ids; int32_t* poly_counts; float* centroids; float* areas; float* poly_verts;
} pairs_ctx;

static void pairs_body(int64_t i, void* c_) {
  pairs_ctx* c = (pairs_ctx*)c_;
  const float* mn = c->bmin + 3 * i;
  const float* mx = c->bmax + 3 * i;
  int64_t k = c->offs ? c->offs[i] : 0, cnt = 0;
  for (int64_t f = 0; f < c->nf; ++f) {
    const float* b = c->tb + 6 * f;
    if (b[0] > mx[0] || b[3] < mn[0] || b[1] > mx[1] || b[4] < mn[1] || b[2] > mx[2] || b[5] < mn[2]) continue;
    float t[9];
    gather_tri(c->V, c->F, f, t);
    if (!orc_sat(t, mn, mx)) continue;
    float verts[24], cen[3] = {0, 0, 0}, ar = 0;
    int pc = 0;
    if (c->clip && !orc_clip_pair(mn, mx, t, c->eps, verts, &pc, cen, &ar)) continue;
    ++cnt;
    if (!c->offs) continue;
    c->box_ids[k] = i;
    c->face_ids[k] = f;
    if (c->clip) {
      c->poly_counts[k] = pc;
      for (int a = 0; a < 3; ++a) c->centroids[3 * k + a] = cen[a];
      c->areas[k] = ar;
      if (c->poly_verts) memcpy(c->poly_verts + 24 * k, verts, sizeof(verts));
    }
    ++k;
  }
  if (c->counts) c->counts[i] = cnt;
}

/* per box: number of faces passing SAT (clip = 0) or SAT and the clip */
void orc_aabb_pair_counts(const float* V, const int32_t* F, int64_t nf, const float* bmin, const float* bmax, int64_t n,
                          int clip, float eps, int64_t* counts) {
  float* tb = tri_boxes(V, F, nf);
  pairs_ctx c = {V, F, nf, tb, bmin, bmax, clip, eps, counts, NULL, NULL, NULL, NULL, NULL, NULL, NULL};
  par_for(n, 16, pairs_body, &c);
  free(tb);
}

/* the pairs, box i's at offs[i] in face order; clip outputs when clip != 0
 * (poly_verts [.,8,3] nullable) */
void orc_aabb_pairs_fill(const float* V, const int32_t* F, int64_t nf, const float* bmin, const float* bmax, int64_t n,
                         int clip, float eps, const int64_t* offs, int64_t* box_ids, int64_t* face_ids,
                         int32_t* poly_counts, float* centroids, float* areas, float* poly_verts) {
  float* tb = tri_boxes(V, F, nf);
  pairs_ctx c = {V, F, nf, tb, bmin, bmax, clip, eps, NULL, offs, box_ids, face_ids, poly_counts, centroids, areas,
                 poly_verts};
  par_for(n, 16, pairs_body, &c);
  free(tb);
}

typedef struct { const float* mn; const float* mx; const float* tri; float eps; int32_t* counts; } clipb_ctx;
static void clipb_body(int64_t k, void* c_) {
  clipb_ctx* c = (clipb_ctx*)c_;
  float verts[24], cen[3], ar;
  int cnt = 0;
  orc_clip_pair(c->mn + 3 * k, c->mx + 3 * k, c->tri + 9 * k, c->eps, verts, &cnt, cen, &ar);
  c->counts[k] = cnt;
}
/* clipped polygon vertex count of each (box k, triangle k) */
void orc_clip_batch(const float* mn, const float* mx, const float* tri9, int64_t m, float eps, int32_t* counts) {
  clipb_ctx c = {mn, mx, tri9, eps, counts};
  par_for(m, 4096, clipb_body, &c);
}
