/*
 * pxo_impl.h -- body of the CPU oracle, included by pxo.c once per precision.
 *
 * Test infrastructure only (see pxo.h). Before inclusion the includer defines
 *   REAL      float or double
 *   SFX(n)    n##_f32 or n##_f64
 *   C(x)      a literal in REAL precision (x##f or x)
 *   EXPR, SQRTR, FLOORR, FABSR, COPYSIGNR   the libm functions for REAL
 *   SPLAT     the projected-splat struct for REAL
 *
 * Every function follows the reference line by line, and evaluates sums in the
 * order the reference's compiled code does: scalar C++ left to right, and for
 * Eigen's small fixed-size products one coefficient at a time as
 * x0 + (x1 + x2) (Eigen/src/Core/Redux.h redux_novec_unroller halves the
 * range), except 4-vectors of float, which Eigen's SSE path reduces as
 * (x0 + x2) + (x1 + x3) (Eigen/src/Core/arch/SSE/PacketMath.h predux).
 * Citations are to engine/native/cpp/src/splat/ unless stated.
 */

/* ------------------------------------------------------------ small maths */

static REAL SFX(dot3)(REAL a0, REAL b0, REAL a1, REAL b1, REAL a2, REAL b2) {
  return a0 * b0 + (a1 * b1 + a2 * b2);
}

/* Sum of the 4-vector product a.b as Eigen's vectorised float path does. */
static REAL SFX(dot4)(const REAL a[4], const REAL b[4]) {
  const REAL p0 = a[0] * b[0], p1 = a[1] * b[1], p2 = a[2] * b[2], p3 = a[3] * b[3];
  return (p0 + p2) + (p1 + p3);
}

/* C = A * B for row-major A (r x k) and B (k x c), k in {2, 3}. */
static void SFX(matmul)(const REAL* A, const REAL* B, REAL* out, int r, int k, int c) {
  for (int i = 0; i < r; ++i) {
    for (int j = 0; j < c; ++j) {
      REAL v;
      if (k == 3) {
        v = SFX(dot3)(A[i * 3 + 0], B[0 * c + j], A[i * 3 + 1], B[1 * c + j], A[i * 3 + 2],
                      B[2 * c + j]);
      } else {
        v = A[i * 2 + 0] * B[0 * c + j] + A[i * 2 + 1] * B[1 * c + j];
      }
      out[i * c + j] = v;
    }
  }
}

static void SFX(transpose)(const REAL* A, REAL* out, int r, int c) {
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < c; ++j) out[j * r + i] = A[i * c + j];
}

/* Unit quaternion (w, x, y, z) from a raw one: Quaternion::normalized, whose
 * squared norm over the (x, y, z, w) storage reduces as (x^2+z^2)+(y^2+w^2). */
static void SFX(quat_normalized)(const REAL q[4], REAL out[4]) {
  const REAL w = q[0], x = q[1], y = q[2], z = q[3];
  const REAL sq = (x * x + z * z) + (y * y + w * w);
  if (sq > C(0.0)) {
    const REAL norm = SQRTR(sq);
    out[0] = w / norm;
    out[1] = x / norm;
    out[2] = y / norm;
    out[3] = z / norm;
  } else {
    out[0] = w;
    out[1] = x;
    out[2] = y;
    out[3] = z;
  }
}

static REAL SFX(quat_norm)(const REAL q[4]) {
  const REAL w = q[0], x = q[1], y = q[2], z = q[3];
  return SQRTR((x * x + z * z) + (y * y + w * w));
}

/* Quaternion::toRotationMatrix (Eigen/src/Geometry/Quaternion.h) on a unit
 * (w, x, y, z); row-major out. */
static void SFX(quat_to_matrix)(const REAL q[4], REAL R[9]) {
  const REAL w = q[0], x = q[1], y = q[2], z = q[3];
  const REAL tx = C(2.0) * x, ty = C(2.0) * y, tz = C(2.0) * z;
  const REAL twx = tx * w, twy = ty * w, twz = tz * w;
  const REAL txx = tx * x, txy = ty * x, txz = tz * x;
  const REAL tyy = ty * y, tyz = tz * y, tzz = tz * z;
  R[0] = C(1.0) - (tyy + tzz);
  R[1] = txy - twz;
  R[2] = txz + twy;
  R[3] = txy + twz;
  R[4] = C(1.0) - (txx + tzz);
  R[5] = tyz - twx;
  R[6] = txz - twy;
  R[7] = tyz + twx;
  R[8] = C(1.0) - (txx + tyy);
}

#define PXO_P(S) (14 + 3 * (S))
#define PAR(c, g) params[(size_t)(c) * (size_t)n + (size_t)(g)]

static void SFX(load_quat)(const REAL* params, int32_t n, int32_t g, REAL q[4]) {
  for (int a = 0; a < 4; ++a) q[a] = PAR(6 + a, g);
}

/* rotationOf + covariance3d (SplatRaster.cpp:78-87): R, scale and Sigma. */
static void SFX(covariance3d)(const REAL* params, int32_t n, int32_t g, REAL R[9], REAL s[3],
                              REAL cov[9]) {
  REAL q[4], qn[4];
  SFX(load_quat)(params, n, g, q);
  SFX(quat_normalized)(q, qn);
  SFX(quat_to_matrix)(qn, R);
  for (int a = 0; a < 3; ++a) s[a] = EXPR(PAR(3 + a, g));
  REAL M[9], Mt[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) M[i * 3 + j] = R[i * 3 + j] * s[j];
  SFX(transpose)(M, Mt, 3, 3);
  SFX(matmul)(M, Mt, cov, 3, 3, 3);
}

/* projectionJacobian (SplatRaster.cpp:91-102), row-major 2x3. */
static void SFX(projection_jacobian)(const REAL p[3], REAL fx, REAL fy, REAL tan_half_x,
                                     REAL tan_half_y, REAL J[6]) {
  const REAL z = p[2];
  const REAL limit_x = tan_half_x * C(1.3);
  const REAL limit_y = tan_half_y * C(1.3);
  REAL ux = p[0] / z, uy = p[1] / z;
  /* std::clamp(v, lo, hi): v < lo ? lo : (hi < v ? hi : v) */
  ux = ux < -limit_x ? -limit_x : (limit_x < ux ? limit_x : ux);
  uy = uy < -limit_y ? -limit_y : (limit_y < uy ? limit_y : uy);
  const REAL x = ux * z, y = uy * z;
  J[0] = fx / z;
  J[1] = C(0.0);
  J[2] = -fx * x / (z * z);
  J[3] = C(0.0);
  J[4] = fy / z;
  J[5] = -fy * y / (z * z);
}

/* shBasis (SplatRaster.cpp:29-52). */
static int SFX(sh_basis)(int degree, const REAL d[3], REAL* basis) {
  const REAL C1 = C(0.4886025119029199);
  const REAL C20 = C(1.0925484305920792), C21 = C(-1.0925484305920792),
             C22 = C(0.31539156525252005), C23 = C(-1.0925484305920792),
             C24 = C(0.5462742152960396);
  const REAL C30 = C(-0.5900435899266435), C31 = C(2.890611442640554),
             C32 = C(-0.4570457994644658), C33 = C(0.3731763325901154),
             C34 = C(-0.4570457994644658), C35 = C(1.445305721320277),
             C36 = C(-0.5900435899266435);
  if (degree < 1) return 0;
  const REAL x = d[0], y = d[1], z = d[2];
  basis[0] = -C1 * y;
  basis[1] = C1 * z;
  basis[2] = -C1 * x;
  if (degree < 2) return 3;
  const REAL xx = x * x, yy = y * y, zz = z * z;
  const REAL xy = x * y, yz = y * z, xz = x * z;
  basis[3] = C20 * xy;
  basis[4] = C21 * yz;
  basis[5] = C22 * (C(2.0) * zz - xx - yy);
  basis[6] = C23 * xz;
  basis[7] = C24 * (xx - yy);
  if (degree < 3) return 8;
  basis[8] = C30 * y * (C(3.0) * xx - yy);
  basis[9] = C31 * xy * z;
  basis[10] = C32 * y * (C(4.0) * zz - xx - yy);
  basis[11] = C33 * z * (C(2.0) * zz - C(3.0) * xx - C(3.0) * yy);
  basis[12] = C34 * x * (C(4.0) * zz - xx - yy);
  basis[13] = C35 * z * (xx - yy);
  basis[14] = C36 * x * (xx - C(3.0) * yy);
  return 15;
}

/* shBasisJacobian (SplatRaster.cpp:55-76): jac[b*3 + axis]. A scalar times a
 * Vec3f multiplies each component. */
static void SFX(sh_basis_jacobian)(int count, const REAL d[3], REAL* jac) {
  const REAL C1 = C(0.4886025119029199);
  const REAL C20 = C(1.0925484305920792), C21 = C(-1.0925484305920792),
             C22 = C(0.31539156525252005), C23 = C(-1.0925484305920792),
             C24 = C(0.5462742152960396);
  const REAL C30 = C(-0.5900435899266435), C31 = C(2.890611442640554),
             C32 = C(-0.4570457994644658), C33 = C(0.3731763325901154),
             C34 = C(-0.4570457994644658), C35 = C(1.445305721320277),
             C36 = C(-0.5900435899266435);
  if (count < 1) return;
  const REAL x = d[0], y = d[1], z = d[2];
#define SETJ(b, cc, a0, a1, a2) \
  do {                          \
    jac[(b)*3 + 0] = (cc) * (a0); \
    jac[(b)*3 + 1] = (cc) * (a1); \
    jac[(b)*3 + 2] = (cc) * (a2); \
  } while (0)
  jac[0] = C(0.0); jac[1] = -C1; jac[2] = C(0.0);
  jac[3] = C(0.0); jac[4] = C(0.0); jac[5] = C1;
  jac[6] = -C1; jac[7] = C(0.0); jac[8] = C(0.0);
  if (count < 8) return;
  const REAL xx = x * x, yy = y * y, zz = z * z;
  SETJ(3, C20, y, x, C(0.0));
  SETJ(4, C21, C(0.0), z, y);
  SETJ(5, C22, C(-2.0) * x, C(-2.0) * y, C(4.0) * z);
  SETJ(6, C23, z, C(0.0), x);
  SETJ(7, C24, C(2.0) * x, C(-2.0) * y, C(0.0));
  if (count < 15) return;
  SETJ(8, C30, C(6.0) * x * y, C(3.0) * xx - C(3.0) * yy, C(0.0));
  SETJ(9, C31, y * z, x * z, x * y);
  SETJ(10, C32, C(-2.0) * x * y, C(4.0) * zz - xx - C(3.0) * yy, C(8.0) * y * z);
  SETJ(11, C33, C(-6.0) * x * z, C(-6.0) * y * z, C(6.0) * zz - C(3.0) * xx - C(3.0) * yy);
  SETJ(12, C34, C(4.0) * zz - C(3.0) * xx - yy, C(-2.0) * x * y, C(8.0) * x * z);
  SETJ(13, C35, C(2.0) * x * z, C(-2.0) * y * z, xx - yy);
  SETJ(14, C36, C(3.0) * xx - C(3.0) * yy, C(-6.0) * x * y, C(0.0));
#undef SETJ
}

/* Vec3f::normalized: d / sqrt(x^2 + (y^2 + z^2)) when nonzero. */
static void SFX(normalized3)(const REAL v[3], REAL out[3]) {
  const REAL sq = v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]);
  if (sq > C(0.0)) {
    const REAL norm = SQRTR(sq);
    out[0] = v[0] / norm;
    out[1] = v[1] / norm;
    out[2] = v[2] / norm;
  } else {
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
  }
}

/* evaluateSh (SplatRaster.cpp:179-199). */
static void SFX(evaluate_sh_internal)(const REAL* params, int32_t n, int32_t g,
                                      int32_t rest_per_channel, int32_t degree,
                                      const REAL direction[3], REAL color[3],
                                      uint32_t* clamped) {
  const REAL C0 = C(0.28209479177387814);
  for (int c = 0; c < 3; ++c) color[c] = C(0.5) + C0 * PAR(11 + c, g);
  REAL basis[15];
  const int count = SFX(sh_basis)(degree, direction, basis);
  const int stride = rest_per_channel;
  const int usable = count < stride ? count : stride;
  for (int c = 0; c < 3; ++c) {
    REAL sum = C(0.0);
    for (int k = 0; k < usable; ++k) sum += basis[k] * PAR(14 + c * stride + k, g);
    color[c] += sum;
  }
  uint32_t flags = 0;
  for (int c = 0; c < 3; ++c) {
    if (color[c] < C(0.0)) {
      flags |= 1u << c;
      color[c] = C(0.0);
    }
  }
  if (clamped) *clamped = flags;
}

static int SFX(splat_cmp)(const void* a, const void* b) {
  const SPLAT* x = (const SPLAT*)a;
  const SPLAT* y = (const SPLAT*)b;
  if (x->depth < y->depth) return -1;
  if (y->depth < x->depth) return 1;
  return x->index < y->index ? -1 : (x->index > y->index ? 1 : 0);
}

/* projectSplats (SplatRaster.cpp:201-263). The reference orders equal depths
 * with std::sort (unspecified); here ties go by gaussian index. */
static int32_t SFX(project_internal)(const REAL* params, int32_t n, int32_t rest_per_channel,
                                     int32_t cloud_sh_degree, const pxs_camera* cam,
                                     const pxs_raster_options* opt, SPLAT* out) {
  REAL W[9], t[3], center[3];
  for (int i = 0; i < 9; ++i) W[i] = cam->R[i];
  for (int i = 0; i < 3; ++i) {
    t[i] = cam->t[i];
    center[i] = cam->center[i];
  }
  const REAL fx = cam->fx, fy = cam->fy, cx = cam->cx, cy = cam->cy;
  const REAL tan_half_x = cam->tan_half_x, tan_half_y = cam->tan_half_y;
  const int degree = opt->sh_degree < cloud_sh_degree ? opt->sh_degree : cloud_sh_degree;
  int32_t count = 0;
  for (int32_t g = 0; g < n; ++g) {
    REAL pos[3] = {PAR(0, g), PAR(1, g), PAR(2, g)};
    REAL p[3];
    for (int i = 0; i < 3; ++i)
      p[i] = SFX(dot3)(W[i * 3 + 0], pos[0], W[i * 3 + 1], pos[1], W[i * 3 + 2], pos[2]) + t[i];
    if (p[2] < C(0.01)) continue;

    REAL J[6], T[6], R[9], s[3], Sigma[9], TS[6], Tt[6], cov[4];
    SFX(projection_jacobian)(p, fx, fy, tan_half_x, tan_half_y, J);
    SFX(matmul)(J, W, T, 2, 3, 3);
    SFX(covariance3d)(params, n, g, R, s, Sigma);
    SFX(matmul)(T, Sigma, TS, 2, 3, 3);
    SFX(transpose)(T, Tt, 2, 3);
    SFX(matmul)(TS, Tt, cov, 2, 3, 2);
    cov[0] += (REAL)opt->screen_dilation;
    cov[3] += (REAL)opt->screen_dilation;

    const REAL det = cov[0] * cov[3] - cov[1] * cov[2];
    if (det <= C(1e-12)) continue;

    SPLAT sp;
    memset(&sp, 0, sizeof(sp));
    sp.index = g;
    sp.mean[0] = fx * p[0] / p[2] + cx;
    sp.mean[1] = fy * p[1] / p[2] + cy;
    sp.cov2d[0] = cov[0];
    sp.cov2d[1] = cov[1];
    sp.cov2d[2] = cov[3];
    sp.conic[0] = cov[3] / det;
    sp.conic[1] = -cov[1] / det;
    sp.conic[2] = cov[0] / det;
    sp.depth = p[2];
    const REAL mid = C(0.5) * (cov[0] + cov[3]);
    const REAL under = mid * mid - det;
    const REAL spread = SQRTR(C(0.0) < under ? under : C(0.0));
    const REAL major = mid + spread;
    sp.radius = C(3.0) * SQRTR(major < C(1e-6) ? C(1e-6) : major);

    if (sp.mean[0] + sp.radius < C(0.0) || sp.mean[0] - sp.radius >= (REAL)cam->width ||
        sp.mean[1] + sp.radius < C(0.0) || sp.mean[1] - sp.radius >= (REAL)cam->height) {
      continue;
    }
    sp.opacity = C(1.0) / (C(1.0) + EXPR(-PAR(10, g)));
    if (sp.opacity < (REAL)opt->min_alpha) continue;

    REAL offset[3], direction[3];
    for (int i = 0; i < 3; ++i) offset[i] = pos[i] - center[i];
    SFX(normalized3)(offset, direction);
    SFX(evaluate_sh_internal)(params, n, g, rest_per_channel, degree, direction, sp.color,
                              &sp.clamped);
    out[count++] = sp;
  }
  qsort(out, (size_t)count, sizeof(SPLAT), SFX(splat_cmp));
  return count;
}

/* tileRange (SplatRaster.cpp:121-126). */
static void SFX(tile_range)(const SPLAT* s, int cols, int rows, int* x0, int* x1, int* y0,
                            int* y1) {
  const REAL tile = (REAL)16;
  int v;
  v = (int)FLOORR((s->mean[0] - s->radius) / tile);
  *x0 = v > 0 ? v : 0;
  v = (int)FLOORR((s->mean[0] + s->radius) / tile);
  *x1 = v < cols - 1 ? v : cols - 1;
  v = (int)FLOORR((s->mean[1] - s->radius) / tile);
  *y0 = v > 0 ? v : 0;
  v = (int)FLOORR((s->mean[1] + s->radius) / tile);
  *y1 = v < rows - 1 ? v : rows - 1;
}

/* buildTiles (SplatRaster.cpp:114-151): counting sort of (tile, splat) pairs,
 * each tile's span in `projected` order. */
static int64_t SFX(build_tiles_internal)(const SPLAT* projected, int32_t count, int32_t width,
                                         int32_t height, int32_t* offsets, int32_t* entries,
                                         int64_t capacity) {
  const int cols = (width + 15) / 16, rows = (height + 15) / 16;
  const int tiles = cols * rows;
  for (int i = 0; i <= tiles; ++i) offsets[i] = 0;
  for (int32_t i = 0; i < count; ++i) {
    int x0, x1, y0, y1;
    SFX(tile_range)(&projected[i], cols, rows, &x0, &x1, &y0, &y1);
    for (int ty = y0; ty <= y1; ++ty)
      for (int tx = x0; tx <= x1; ++tx) offsets[ty * cols + tx + 1]++;
  }
  for (int i = 0; i < tiles; ++i) offsets[i + 1] += offsets[i];
  const int64_t total = offsets[tiles];
  if (total > capacity) return total;
  int32_t* cursor = (int32_t*)malloc(sizeof(int32_t) * (size_t)(tiles > 0 ? tiles : 1));
  for (int i = 0; i < tiles; ++i) cursor[i] = offsets[i];
  for (int32_t i = 0; i < count; ++i) {
    int x0, x1, y0, y1;
    SFX(tile_range)(&projected[i], cols, rows, &x0, &x1, &y0, &y1);
    for (int ty = y0; ty <= y1; ++ty)
      for (int tx = x0; tx <= x1; ++tx) entries[cursor[ty * cols + tx]++] = i;
  }
  free(cursor);
  return total;
}

/* Per-pixel power -0.5 (a dx^2 + c dy^2) - b dx dy (SplatRaster.cpp:295-297). */
static REAL SFX(power)(const SPLAT* s, REAL dx, REAL dy) {
  return C(-0.5) * (s->conic[0] * dx * dx + s->conic[2] * dy * dy) - s->conic[1] * dx * dy;
}

/* rasterizeSplats (SplatRaster.cpp:265-315). */
static void SFX(rasterize_internal)(const SPLAT* projected, int32_t count,
                                    const pxs_camera* cam, const pxs_raster_options* opt,
                                    REAL* rgb, REAL* transmittance) {
  const int width = cam->width, height = cam->height;
  const size_t pixels = (size_t)width * (size_t)height;
  for (size_t i = 0; i < pixels * 3; ++i) rgb[i] = C(0.0);
  if (transmittance)
    for (size_t i = 0; i < pixels; ++i) transmittance[i] = C(1.0);
  if (pixels == 0) return;
  const int cols = (width + 15) / 16, rows = (height + 15) / 16;
  const int tiles = cols * rows;
  int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(tiles + 1));
  int64_t total = SFX(build_tiles_internal)(projected, count, width, height, offsets, NULL, 0);
  int32_t* entries = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  SFX(build_tiles_internal)(projected, count, width, height, offsets, entries, total);
  const REAL max_alpha = C(0.99);
  for (int ty = 0; ty < rows; ++ty) {
    for (int tx = 0; tx < cols; ++tx) {
      const int tile = ty * cols + tx;
      const int begin = offsets[tile], end = offsets[tile + 1];
      const int y_end = height < (ty + 1) * 16 ? height : (ty + 1) * 16;
      const int x_end = width < (tx + 1) * 16 ? width : (tx + 1) * 16;
      for (int y = ty * 16; y < y_end; ++y) {
        for (int x = tx * 16; x < x_end; ++x) {
          const size_t pixel = (size_t)y * (size_t)width + (size_t)x;
          const REAL px = (REAL)x + C(0.5), py = (REAL)y + C(0.5);
          REAL T = C(1.0);
          REAL acc[3] = {C(0.0), C(0.0), C(0.0)};
          for (int e = begin; e < end; ++e) {
            const SPLAT* s = &projected[entries[e]];
            const REAL dx = px - s->mean[0], dy = py - s->mean[1];
            const REAL power = SFX(power)(s, dx, dy);
            if (power > C(0.0)) continue;
            REAL alpha = s->opacity * EXPR(power);
            alpha = alpha < max_alpha ? alpha : max_alpha; /* std::min(kMaxAlpha, .) */
            if (alpha < (REAL)opt->min_alpha) continue;
            for (int c = 0; c < 3; ++c) acc[c] += T * alpha * s->color[c];
            T *= C(1.0) - alpha;
            if (T < (REAL)opt->transmittance_cutoff) break;
          }
          for (int c = 0; c < 3; ++c) rgb[pixel * 3 + c] = acc[c] + T * (REAL)opt->background[c];
          if (transmittance) transmittance[pixel] = T;
        }
      }
    }
  }
  free(entries);
  free(offsets);
}

/* rasterizeSplatsBackward (SplatRaster.cpp:322-576). */
static void SFX(backward_internal)(const REAL* params, int32_t n, int32_t rest_per_channel,
                                   int32_t cloud_sh_degree, const pxs_camera* cam,
                                   const pxs_raster_options* opt, const SPLAT* projected,
                                   int32_t count, const REAL* dL_drgb, REAL* grads,
                                   REAL* screen_gradient, int32_t* visible_count) {
  const int width = cam->width, height = cam->height;
  if (count == 0 || width == 0) return;
  const size_t cnt = (size_t)count;
  REAL* dmean = (REAL*)calloc(cnt * 2, sizeof(REAL));
  REAL* dconic = (REAL*)calloc(cnt * 3, sizeof(REAL));
  REAL* dopacity = (REAL*)calloc(cnt, sizeof(REAL));
  REAL* dcolor = (REAL*)calloc(cnt * 3, sizeof(REAL));
  REAL* dmean_abs = (REAL*)calloc(cnt, sizeof(REAL));
  int* touched = (int*)calloc(cnt, sizeof(int));

  const int cols = (width + 15) / 16, rows = (height + 15) / 16;
  const int tiles = cols * rows;
  int32_t* offsets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(tiles + 1));
  int64_t total = SFX(build_tiles_internal)(projected, count, width, height, offsets, NULL, 0);
  int32_t* entries = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
  SFX(build_tiles_internal)(projected, count, width, height, offsets, entries, total);
  const REAL max_alpha = C(0.99);
  const REAL min_alpha = (REAL)opt->min_alpha;

  for (int ty = 0; ty < rows; ++ty) {
    for (int tx = 0; tx < cols; ++tx) {
      const int tile = ty * cols + tx;
      const int begin = offsets[tile], end = offsets[tile + 1];
      const int y_end = height < (ty + 1) * 16 ? height : (ty + 1) * 16;
      const int x_end = width < (tx + 1) * 16 ? width : (tx + 1) * 16;
      for (int y = ty * 16; y < y_end; ++y) {
        for (int x = tx * 16; x < x_end; ++x) {
          const size_t pixel = (size_t)y * (size_t)width + (size_t)x;
          const REAL px = (REAL)x + C(0.5), py = (REAL)y + C(0.5);
          const REAL* dLp = &dL_drgb[pixel * 3];
          REAL T = C(1.0);
          int last = begin;
          for (int e = begin; e < end; ++e) {
            const SPLAT* s = &projected[entries[e]];
            const REAL dx = px - s->mean[0], dy = py - s->mean[1];
            const REAL power = SFX(power)(s, dx, dy);
            if (power > C(0.0)) continue;
            REAL alpha = s->opacity * EXPR(power);
            alpha = alpha < max_alpha ? alpha : max_alpha;
            if (alpha < min_alpha) continue;
            T *= C(1.0) - alpha;
            last = e + 1;
            if (T < (REAL)opt->transmittance_cutoff) break;
          }
          const REAL final_T = T;
          REAL suffix[3] = {C(0.0), C(0.0), C(0.0)};
          REAL last_alpha = C(0.0);
          REAL last_color[3] = {C(0.0), C(0.0), C(0.0)};
          REAL background_term = C(0.0);
          for (int c = 0; c < 3; ++c) background_term += (REAL)opt->background[c] * dLp[c];
          for (int e = last - 1; e >= begin; --e) {
            const size_t si = (size_t)entries[e];
            const SPLAT* s = &projected[si];
            const REAL dx = px - s->mean[0], dy = py - s->mean[1];
            const REAL power = SFX(power)(s, dx, dy);
            if (power > C(0.0)) continue;
            const REAL gw = EXPR(power);
            const REAL raw_alpha = s->opacity * gw;
            const REAL alpha = raw_alpha < max_alpha ? raw_alpha : max_alpha;
            if (alpha < min_alpha) continue;
            T /= C(1.0) - alpha;
            const REAL weight = alpha * T;
            REAL dL_dalpha = C(0.0);
            for (int c = 0; c < 3; ++c) {
              dcolor[si * 3 + c] += weight * dLp[c];
              suffix[c] = last_alpha * last_color[c] + (C(1.0) - last_alpha) * suffix[c];
              last_color[c] = s->color[c];
              dL_dalpha += (s->color[c] - suffix[c]) * T * dLp[c];
            }
            last_alpha = alpha;
            dL_dalpha += -final_T / (C(1.0) - alpha) * background_term;
            if (raw_alpha >= max_alpha) continue;
            dopacity[si] += gw * dL_dalpha;
            const REAL dL_dweight = s->opacity * dL_dalpha;
            const REAL gx = gw * dx, gy = gw * dy;
            const REAL dm0 = dL_dweight * (-gx * s->conic[0] - gy * s->conic[1]);
            const REAL dm1 = dL_dweight * (-gy * s->conic[2] - gx * s->conic[1]);
            dmean[si * 2 + 0] -= dm0;
            dmean[si * 2 + 1] -= dm1;
            dmean_abs[si] += SQRTR(dm0 * dm0 + dm1 * dm1);
            dconic[si * 3 + 0] += C(-0.5) * dL_dweight * gx * dx;
            dconic[si * 3 + 1] += C(-1.0) * dL_dweight * gx * dy;
            dconic[si * 3 + 2] += C(-0.5) * dL_dweight * gy * dy;
            touched[si] = 1;
          }
        }
      }
    }
  }
  free(entries);
  free(offsets);

  /* screen space back to the parameters (SplatRaster.cpp:437-575) */
  REAL W[9], Wt[9], t[3], center[3];
  for (int i = 0; i < 9; ++i) W[i] = cam->R[i];
  SFX(transpose)(W, Wt, 3, 3);
  for (int i = 0; i < 3; ++i) {
    t[i] = cam->t[i];
    center[i] = cam->center[i];
  }
  const REAL fx = cam->fx, fy = cam->fy;
  const REAL tan_half_x = cam->tan_half_x, tan_half_y = cam->tan_half_y;
  const int rest_stride = 3 * rest_per_channel;
  const REAL C0 = C(0.28209479177387814);
  const REAL slack = C(1.3);

  for (size_t si = 0; si < cnt; ++si) {
    const SPLAT* s = &projected[si];
    const int32_t g = s->index;
    visible_count[g] += 1;
    screen_gradient[g] += dmean_abs[si];
    if (touched[si] == 0) continue;
#define GR(c) grads[(size_t)(c) * (size_t)n + (size_t)g]
    const REAL opacity = s->opacity;
    GR(10) += dopacity[si] * opacity * (C(1.0) - opacity);

    REAL dcol[3];
    for (int c = 0; c < 3; ++c) {
      dcol[c] = dcolor[si * 3 + c];
      if (s->clamped & (1u << c)) dcol[c] = C(0.0);
      GR(11 + c) += C0 * dcol[c];
    }

    REAL ddir[3] = {C(0.0), C(0.0), C(0.0)};
    const int degree = opt->sh_degree < cloud_sh_degree ? opt->sh_degree : cloud_sh_degree;
    const int per_channel = rest_stride / 3;
    const REAL pos[3] = {PAR(0, g), PAR(1, g), PAR(2, g)};
    REAL offset[3];
    for (int i = 0; i < 3; ++i) offset[i] = pos[i] - center[i];
    const REAL distance =
        SQRTR(offset[0] * offset[0] + (offset[1] * offset[1] + offset[2] * offset[2]));
    if (degree >= 1 && distance > C(1e-9) && per_channel > 0) {
      REAL direction[3], basis[15], jac[45];
      for (int i = 0; i < 3; ++i) direction[i] = offset[i] / distance;
      const int basis_count = SFX(sh_basis)(degree, direction, basis);
      const int usable = basis_count < per_channel ? basis_count : per_channel;
      SFX(sh_basis_jacobian)(basis_count, direction, jac);
      for (int c = 0; c < 3; ++c) {
        if (dcol[c] == C(0.0)) continue;
        for (int b = 0; b < usable; ++b) {
          GR(14 + c * per_channel + b) += basis[b] * dcol[c];
          const REAL k = PAR(14 + c * per_channel + b, g) * dcol[c];
          for (int a = 0; a < 3; ++a) ddir[a] += jac[b * 3 + a] * k;
        }
      }
    }

    REAL p[3];
    for (int i = 0; i < 3; ++i)
      p[i] = SFX(dot3)(W[i * 3 + 0], pos[0], W[i * 3 + 1], pos[1], W[i * 3 + 2], pos[2]) + t[i];
    const REAL z = p[2];
    const REAL dmx = dmean[si * 2 + 0], dmy = dmean[si * 2 + 1];
    REAL dp[3] = {fx / z * dmx, fy / z * dmy, -(fx * p[0] * dmx + fy * p[1] * dmy) / (z * z)};

    /* conic -> 2D covariance: -(A D A) with D the symmetric gradient */
    const REAL A[4] = {s->conic[0], s->conic[1], s->conic[1], s->conic[2]};
    const REAL D[4] = {dconic[si * 3 + 0], C(0.5) * dconic[si * 3 + 1],
                       C(0.5) * dconic[si * 3 + 1], dconic[si * 3 + 2]};
    REAL AD[4], ADA[4], dcov2[4];
    SFX(matmul)(A, D, AD, 2, 2, 2);
    SFX(matmul)(AD, A, ADA, 2, 2, 2);
    for (int i = 0; i < 4; ++i) dcov2[i] = -ADA[i];

    REAL J[6], T[6], Tt[6], R[9], sc[3], Sigma[9];
    SFX(projection_jacobian)(p, fx, fy, tan_half_x, tan_half_y, J);
    SFX(matmul)(J, W, T, 2, 3, 3);
    SFX(covariance3d)(params, n, g, R, sc, Sigma);
    /* dL_dcov3d = T^T dcov2 T */
    REAL TtD[6], dcov3[9];
    SFX(transpose)(T, Tt, 2, 3);
    SFX(matmul)(Tt, dcov2, TtD, 3, 2, 2);
    SFX(matmul)(TtD, T, dcov3, 3, 2, 3);
    /* dL_dT = ((2 dcov2) T) Sigma; dL_dJ = dL_dT W^T */
    REAL D2[4], D2T[6], dT[6], dJ[6];
    for (int i = 0; i < 4; ++i) D2[i] = C(2.0) * dcov2[i];
    SFX(matmul)(D2, T, D2T, 2, 2, 3);
    SFX(matmul)(D2T, Sigma, dT, 2, 3, 3);
    SFX(matmul)(dT, Wt, dJ, 2, 3, 3);

    const int clamped_x = FABSR(p[0] / z) > tan_half_x * slack;
    const int clamped_y = FABSR(p[1] / z) > tan_half_y * slack;
    const REAL lim_x = tan_half_x * slack, lim_y = tan_half_y * slack;
    const REAL jx = clamped_x ? COPYSIGNR(lim_x, p[0]) * z : p[0];
    const REAL jy = clamped_y ? COPYSIGNR(lim_y, p[1]) * z : p[1];
    if (!clamped_x) dp[0] += dJ[2] * (-fx / (z * z));
    if (!clamped_y) dp[1] += dJ[5] * (-fy / (z * z));
    const REAL dz_x = (clamped_x ? C(1.0) : C(2.0)) * fx * jx / (z * z * z);
    const REAL dz_y = (clamped_y ? C(1.0) : C(2.0)) * fy * jy / (z * z * z);
    dp[2] += dJ[0] * (-fx / (z * z)) + dJ[4] * (-fy / (z * z)) + dJ[2] * dz_x + dJ[5] * dz_y;

    REAL dpos[3];
    for (int i = 0; i < 3; ++i)
      dpos[i] = SFX(dot3)(Wt[i * 3 + 0], dp[0], Wt[i * 3 + 1], dp[1], Wt[i * 3 + 2], dp[2]);
    const REAL ddir_sq = ddir[0] * ddir[0] + (ddir[1] * ddir[1] + ddir[2] * ddir[2]);
    if (distance > C(1e-9) && ddir_sq > C(0.0)) {
      REAL direction[3];
      for (int i = 0; i < 3; ++i) direction[i] = offset[i] / distance;
      const REAL dd = SFX(dot3)(direction[0], ddir[0], direction[1], ddir[1], direction[2],
                                ddir[2]);
      for (int i = 0; i < 3; ++i) dpos[i] += (ddir[i] - direction[i] * dd) / distance;
    }
    for (int i = 0; i < 3; ++i) GR(i) += dpos[i];

    /* Sigma = (R S)(R S)^T -> scale and rotation */
    REAL M[9], sym[9], sym2[9], dM[9], dS[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i * 3 + j] = R[i * 3 + j] * sc[j];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) sym[i * 3 + j] = C(0.5) * (dcov3[i * 3 + j] + dcov3[j * 3 + i]);
    for (int i = 0; i < 9; ++i) sym2[i] = C(2.0) * sym[i];
    SFX(matmul)(sym2, M, dM, 3, 3, 3);
    REAL Rt[9];
    SFX(transpose)(R, Rt, 3, 3);
    SFX(matmul)(Rt, dM, dS, 3, 3, 3);
    for (int a = 0; a < 3; ++a) GR(3 + a) += dS[a * 3 + a] * sc[a];

    REAL dR[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) dR[r * 3 + c] = dM[r * 3 + c] * sc[c];
    REAL qraw[4], q[4];
    SFX(load_quat)(params, n, g, qraw);
    REAL raw_norm = SFX(quat_norm)(qraw);
    raw_norm = raw_norm < C(1e-12) ? C(1e-12) : raw_norm;
    SFX(quat_normalized)(qraw, q);
    const REAL qw = q[0], qx = q[1], qy = q[2], qz = q[3];
#define dRm(r, c) dR[(r)*3 + (c)]
    REAL dq[4];
    dq[0] = C(0.0) + C(2.0) * (-qz * dRm(0, 1) + qy * dRm(0, 2) + qz * dRm(1, 0) -
                               qx * dRm(1, 2) - qy * dRm(2, 0) + qx * dRm(2, 1));
    dq[1] = C(0.0) + C(2.0) * (qy * dRm(0, 1) + qz * dRm(0, 2) + qy * dRm(1, 0) -
                               C(2.0) * qx * dRm(1, 1) - qw * dRm(1, 2) + qz * dRm(2, 0) +
                               qw * dRm(2, 1) - C(2.0) * qx * dRm(2, 2));
    dq[2] = C(0.0) + C(2.0) * (C(-2.0) * qy * dRm(0, 0) + qx * dRm(0, 1) + qw * dRm(0, 2) +
                               qx * dRm(1, 0) + qz * dRm(1, 2) - qw * dRm(2, 0) +
                               qz * dRm(2, 1) - C(2.0) * qy * dRm(2, 2));
    dq[3] = C(0.0) + C(2.0) * (C(-2.0) * qz * dRm(0, 0) - qw * dRm(0, 1) + qx * dRm(0, 2) +
                               qw * dRm(1, 0) - C(2.0) * qz * dRm(1, 1) + qy * dRm(1, 2) +
                               qx * dRm(2, 0) + qy * dRm(2, 1));
#undef dRm
    const REAL unit[4] = {qw, qx, qy, qz};
    const REAL ud = SFX(dot4)(unit, dq);
    for (int a = 0; a < 4; ++a) GR(6 + a) += (dq[a] - unit[a] * ud) / raw_norm;
#undef GR
  }
  free(dmean);
  free(dconic);
  free(dopacity);
  free(dcolor);
  free(dmean_abs);
  free(touched);
}

/* ------------------------------------------------------------------ loss */

/* ssimKernel (SplatRaster.cpp:587-600): 11 taps, sigma 1.5, normalised. */
static void SFX(ssim_kernel)(REAL k[11]) {
  REAL total = C(0.0);
  for (int i = -5; i <= 5; ++i) {
    const REAL v = EXPR(C(-0.5) * (REAL)(i * i) / (C(1.5) * C(1.5)));
    k[i + 5] = v;
    total += v;
  }
  for (int i = 0; i < 11; ++i) k[i] /= total;
}

/* blur (SplatRaster.cpp:614-642): separable, zero padded. */
static void SFX(blur)(const REAL* src, int width, int height, REAL* tmp, REAL* dst,
                      const REAL k[11]) {
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      REAL sum = C(0.0);
      for (int i = -5; i <= 5; ++i) {
        const int sx = x + i;
        if (sx < 0 || sx >= width) continue;
        sum += k[i + 5] * src[(size_t)y * width + sx];
      }
      tmp[(size_t)y * width + x] = sum;
    }
  }
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      REAL sum = C(0.0);
      for (int i = -5; i <= 5; ++i) {
        const int sy = y + i;
        if (sy < 0 || sy >= height) continue;
        sum += k[i + 5] * tmp[(size_t)sy * width + x];
      }
      dst[(size_t)y * width + x] = sum;
    }
  }
}

/* meanSsim (SplatRaster.cpp:646-710). */
static REAL SFX(mean_ssim_internal)(const REAL* rendered, const REAL* target, int width,
                                    int height, REAL* d_rendered) {
  const size_t pixels = (size_t)width * (size_t)height;
  if (pixels == 0) return C(0.0);
  if (d_rendered)
    for (size_t i = 0; i < pixels * 3; ++i) d_rendered[i] = C(0.0);
  REAL k[11];
  SFX(ssim_kernel)(k);
  const REAL scale = C(1.0) / (REAL)(pixels * 3);
  const REAL c1 = C(0.01) * C(0.01), c2 = C(0.03) * C(0.03);
  REAL total = C(0.0);
  REAL* buf = (REAL*)malloc(sizeof(REAL) * pixels * 16);
  REAL *x = buf, *y = buf + pixels, *xx = buf + 2 * pixels, *yy = buf + 3 * pixels,
       *xy = buf + 4 * pixels, *mu_x = buf + 5 * pixels, *mu_y = buf + 6 * pixels,
       *exx = buf + 7 * pixels, *eyy = buf + 8 * pixels, *exy = buf + 9 * pixels,
       *t_mu = buf + 10 * pixels, *t_var = buf + 11 * pixels, *t_cov = buf + 12 * pixels,
       *blurred = buf + 13 * pixels, *scratch = buf + 14 * pixels, *tmp = buf + 15 * pixels;
  for (int channel = 0; channel < 3; ++channel) {
    for (size_t p = 0; p < pixels; ++p) {
      x[p] = rendered[p * 3 + channel];
      y[p] = target[p * 3 + channel];
      xx[p] = x[p] * x[p];
      yy[p] = y[p] * y[p];
      xy[p] = x[p] * y[p];
    }
    SFX(blur)(x, width, height, tmp, mu_x, k);
    SFX(blur)(y, width, height, tmp, mu_y, k);
    SFX(blur)(xx, width, height, tmp, exx, k);
    SFX(blur)(yy, width, height, tmp, eyy, k);
    SFX(blur)(xy, width, height, tmp, exy, k);
    for (size_t p = 0; p < pixels; ++p) {
      const REAL var_x = exx[p] - mu_x[p] * mu_x[p];
      const REAL var_y = eyy[p] - mu_y[p] * mu_y[p];
      const REAL cov = exy[p] - mu_x[p] * mu_y[p];
      const REAL a = C(2.0) * mu_x[p] * mu_y[p] + c1;
      const REAL b = C(2.0) * cov + c2;
      const REAL c = mu_x[p] * mu_x[p] + mu_y[p] * mu_y[p] + c1;
      const REAL d = var_x + var_y + c2;
      total += (a * b) / (c * d);
      if (!d_rendered) continue;
      t_mu[p] = scale * (C(2.0) * mu_y[p] * b / (c * d) - C(2.0) * mu_x[p] * a * b / (c * c * d));
      t_var[p] = scale * (-(a * b) / (c * d * d));
      t_cov[p] = scale * (C(2.0) * a / (c * d));
    }
    if (!d_rendered) continue;
    SFX(blur)(t_mu, width, height, tmp, blurred, k);
    for (size_t p = 0; p < pixels; ++p) d_rendered[p * 3 + channel] += blurred[p];
    SFX(blur)(t_var, width, height, tmp, blurred, k);
    for (size_t p = 0; p < pixels; ++p) d_rendered[p * 3 + channel] += C(2.0) * x[p] * blurred[p];
    for (size_t p = 0; p < pixels; ++p) scratch[p] = t_var[p] * mu_x[p];
    SFX(blur)(scratch, width, height, tmp, blurred, k);
    for (size_t p = 0; p < pixels; ++p) d_rendered[p * 3 + channel] -= C(2.0) * blurred[p];
    SFX(blur)(t_cov, width, height, tmp, blurred, k);
    for (size_t p = 0; p < pixels; ++p) d_rendered[p * 3 + channel] += y[p] * blurred[p];
    for (size_t p = 0; p < pixels; ++p) scratch[p] = t_cov[p] * mu_y[p];
    SFX(blur)(scratch, width, height, tmp, blurred, k);
    for (size_t p = 0; p < pixels; ++p) d_rendered[p * 3 + channel] -= blurred[p];
  }
  free(buf);
  return total * scale;
}

/* photometricLoss (SplatRaster.cpp:712-738). */
static REAL SFX(photometric_loss_internal)(const REAL* rendered, const REAL* target, int width,
                                           int height, REAL ssim_weight, REAL* dL_drgb) {
  const size_t values = (size_t)width * (size_t)height * 3;
  if (dL_drgb)
    for (size_t i = 0; i < values; ++i) dL_drgb[i] = C(0.0);
  if (values == 0) return C(0.0);
  const REAL inverse = C(1.0) / (REAL)values;
  REAL l1 = C(0.0);
  for (size_t i = 0; i < values; ++i) {
    const REAL diff = rendered[i] - target[i];
    l1 += FABSR(diff);
    if (dL_drgb) {
      const REAL sign = diff > C(0.0) ? C(1.0) : (diff < C(0.0) ? C(-1.0) : C(0.0));
      dL_drgb[i] = (C(1.0) - ssim_weight) * sign * inverse;
    }
  }
  l1 *= inverse;
  if (ssim_weight <= C(0.0)) return l1;
  REAL* d_ssim = dL_drgb ? (REAL*)malloc(sizeof(REAL) * values) : NULL;
  const REAL ssim = SFX(mean_ssim_internal)(rendered, target, width, height, d_ssim);
  if (dL_drgb) {
    for (size_t i = 0; i < values; ++i) dL_drgb[i] -= ssim_weight * d_ssim[i];
    free(d_ssim);
  }
  return (C(1.0) - ssim_weight) * l1 + ssim_weight * (C(1.0) - ssim);
}

#undef PAR
