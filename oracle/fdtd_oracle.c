/*
 * fdtd_oracle.c -- CPU oracle for the FDTD time step, in C with POSIX threads.
 * TEST INFRASTRUCTURE AND CPU BASELINE ONLY: only tests/, __graft_entry__
 * and bench.py's CPU legs load it; the product path never does.
 *
 * The same step as oracle/fdtd_oracle.py (the numpy restatement of the
 * reference fdtdsarsim, pinned bit for bit to the reference's own outputs),
 * with the same evaluation order and precision for every operation, so
 * that both oracles agree bit for bit:
 *   H update   cpu/field_updates.py:198-240
 *   H CPML     cpu/field_updates.py:243-366 (faces z, x, y)
 *   injection  cpu/main_sim.py:147-150 (all x, all y)
 *   E update   cpu/field_updates.py:18-63
 *   E CPML     cpu/field_updates.py:66-191 (faces z, x, y)
 *   injection  cpu/main_sim.py:158-161
 *   phasors    cpu/field_updates.py:373-461 (float64 sum of the stored
 *              value and the float64 term, rounded to the storage type)
 * Build with -ffp-contract=off (no fused multiply-adds, as the reference's
 * numba kernels) and without -ffast-math. Arrays are C-contiguous
 * (nz, ny, nx); CPML auxiliaries as in the numpy oracle: z faces
 * (npml, ny, nx), x faces (nz, ny, npml), y faces (nz, npml, nx).
 */
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>

/* auxiliary slots, numpy names: z faces Exz Eyz Hxz Hyz, x faces Eyx Ezx Hyx
 * Hzx, y faces Exy Ezy Hxy Hzy; [face][side 0 low, 1 high][slot] */
typedef struct oracle_state {
  int nx, ny, nz, npml, tfsf_z;
  int t, nt_inc;
  int dtype;               /* 0 float, 1 double */
  int nthreads;
  double db, dtm0, dte0dx, dx;   /* exactly representable in the element type */
  void *ex, *ey, *ez, *hx, *hy, *hz;
  const void *ca, *cb;
  void *psi[3][2][4];
  const void *prof[8];     /* be_d bh_d ce_d ch_d be_u bh_u ce_u ch_u, npml each */
  const void *inc[4];      /* ex ey hx hy, (nt_inc, ny, nx) */
  void *ph[24];            /* interleaved complex, reference order */
  double ce, se, ch, sh;   /* phase factors of step t */
} oracle_state;

#define IDX(z, y, x) (((size_t)(z) * ny + (y)) * nx + (x))
#define RS __restrict__

#define DEFINE_STEP(T, NAME)                                                           \
__attribute__((target_clones("avx2", "default"))) static void NAME(const oracle_state *s, int phase, int lo, int hi) {                                           \
  const int nx = s->nx, ny = s->ny, nz = s->nz, m = s->npml;                           \
  T *ex = (T *)s->ex, *ey = (T *)s->ey, *ez = (T *)s->ez;                              \
  T *hx = (T *)s->hx, *hy = (T *)s->hy, *hz = (T *)s->hz;                              \
  const T *ca = (const T *)s->ca, *cb = (const T *)s->cb;                              \
  const T Db = (T)s->db, dtm0 = (T)s->dtm0, dte0dx = (T)s->dte0dx, dx = (T)s->dx;      \
  const T *be[2] = {(const T *)s->prof[0], (const T *)s->prof[4]};                     \
  const T *bh[2] = {(const T *)s->prof[1], (const T *)s->prof[5]};                     \
  const T *cE[2] = {(const T *)s->prof[2], (const T *)s->prof[6]};                     \
  const T *cH[2] = {(const T *)s->prof[3], (const T *)s->prof[7]};                     \
  /* ---- phase 0: H main update, planes [lo, hi); per row, the x range of   \
   * each component's update (no branch in the inner loops) ---- */                   \
  if (phase == 0)                                                                      \
  for (int z = lo; z < hi && z < nz - 1; ++z)                                          \
    for (int y = 0; y < ny - 1; ++y) {                                                 \
      const size_t r = IDX(z, y, 0), rz = IDX(z + 1, y, 0), ry = IDX(z, y + 1, 0);     \
      T *RS hxr = hx + r; T *RS hyr = hy + r; T *RS hzr = hz + r;                      \
      const T *RS exr = ex + r; const T *RS eyr = ey + r; const T *RS ezr = ez + r;    \
      const T *RS eyz = ey + rz; const T *RS exz = ex + rz;                            \
      const T *RS ezy = ez + ry; const T *RS exy = ex + ry;                            \
      for (int x = 1; x < nx - 1; ++x)                                                 \
        hxr[x] -= Db * ((ezy[x] - ezr[x]) - (eyz[x] - eyr[x]));                        \
      if (y >= 1)                                                                      \
        for (int x = 0; x < nx - 1; ++x)                                               \
          hyr[x] -= Db * ((exz[x] - exr[x]) - (ezr[x + 1] - ezr[x]));                  \
      if (z >= 1)                                                                      \
        for (int x = 0; x < nx - 1; ++x)                                               \
          hzr[x] -= Db * ((eyr[x + 1] - eyr[x]) - (exy[x] - exr[x]));                  \
    }                                                                                  \
  /* ---- phase 1: H CPML over the face regions only: z faces, then x, then    \
   * y (the reference's kernel order; a cell's corrections keep that order)     \
   * ---- */                                                                            \
  /* phase 7: the z faces, rows of the face planes [lo, hi) (planes           \
   * z < m - 1 and nz - m <= z < nz - 1, (ny - 1) rows each), so that every     \
   * thread gets an equal share; then phase 1: x and y faces per plane */       \
  if (phase == 7)                                                                      \
  for (int w = lo; w < hi; ++w) {                                                      \
    const int j = w / (ny - 1), y = w % (ny - 1);                                      \
    const int sd = j < m - 1 ? 0 : 1, q = sd ? j - (m - 1) : j;                        \
    const int z = sd ? nz - m + q : q;                                                 \
    const T b = bh[sd][q], c = cH[sd][q];                                              \
    const size_t r = IDX(z, y, 0), rz = IDX(z + 1, y, 0);                              \
    T *RS Pyz = (T *)s->psi[0][sd][3] + ((size_t)q * ny + y) * nx;                     \
    T *RS Pxz = (T *)s->psi[0][sd][2] + ((size_t)q * ny + y) * nx;                     \
    T *RS hxr = hx + r; T *RS hyr = hy + r;                                            \
    const T *RS exr = ex + r; const T *RS eyr = ey + r;                                \
    const T *RS exz = ex + rz; const T *RS eyz = ey + rz;                              \
    for (int x = 0; x < nx - 1; ++x) {                                                 \
      Pyz[x] = b * Pyz[x] + c * (exz[x] - exr[x]) / dx;                                \
      Pxz[x] = b * Pxz[x] + c * (eyz[x] - eyr[x]) / dx;                                \
      hyr[x] -= dtm0 * Pyz[x];                                                         \
      hxr[x] += dtm0 * Pxz[x];                                                         \
    }                                                                                  \
  }                                                                                    \
  if (phase == 1)                                                                      \
  for (int z = lo; z < hi && z < nz - 1; ++z) {                                        \
    for (int y = 0; y < ny - 1; ++y)                                                   \
      for (int sx = 0; sx < 2; ++sx) {                                                 \
        const int x0 = sx ? nx - m : 0, x1 = sx ? nx - 1 : m - 1;                      \
        for (int x = x0; x < x1; ++x) {                                                \
          const int qx = sx ? x - (nx - m) : x;                                        \
          const size_t i = IDX(z, y, x);                                               \
          T *Pzx = (T *)s->psi[1][sx][3], *Pyx = (T *)s->psi[1][sx][2];                \
          const size_t k = ((size_t)z * ny + y) * m + qx;                              \
          const T b = bh[sx][qx], c = cH[sx][qx];                                      \
          Pzx[k] = b * Pzx[k] + c * (ey[i + 1] - ey[i]) / dx;                          \
          Pyx[k] = b * Pyx[k] + c * (ez[i + 1] - ez[i]) / dx;                          \
          hz[i] -= dtm0 * Pzx[k];                                                      \
          hy[i] += dtm0 * Pyx[k];                                                      \
        }                                                                              \
      }                                                                                \
    for (int sy = 0; sy < 2; ++sy) {                                                   \
      const int y0 = sy ? ny - m : 0, y1 = sy ? ny - 1 : m - 1;                        \
      for (int y = y0; y < y1; ++y) {                                                  \
        const int qy = sy ? y - (ny - m) : y;                                          \
        const T b = bh[sy][qy], c = cH[sy][qy];                                        \
        const size_t r = IDX(z, y, 0), ry = IDX(z, y + 1, 0);                          \
        T *RS Pxy = (T *)s->psi[2][sy][2] + ((size_t)z * m + qy) * nx;                 \
        T *RS Pzy = (T *)s->psi[2][sy][3] + ((size_t)z * m + qy) * nx;                 \
        T *RS hxr = hx + r; T *RS hzr = hz + r;                                        \
        const T *RS exr = ex + r; const T *RS ezr = ez + r;                            \
        const T *RS exy = ex + ry; const T *RS ezy = ez + ry;                          \
        for (int x = 0; x < nx - 1; ++x) {                                             \
          Pxy[x] = b * Pxy[x] + c * (ezy[x] - ezr[x]) / dx;                            \
          Pzy[x] = b * Pzy[x] + c * (exy[x] - exr[x]) / dx;                            \
          hxr[x] -= dtm0 * Pxy[x];                                                     \
          hzr[x] += dtm0 * Pzy[x];                                                     \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
  }                                                                                    \
  const int inj = s->t < s->nt_inc;                                                    \
  /* ---- phase 2: E-field injection into H, rows [lo, hi) ---- */                     \
  if (phase == 2 && inj) {                                                             \
    const T *iey = (const T *)s->inc[1] + (size_t)s->t * ny * nx;                      \
    const T *iex = (const T *)s->inc[0] + (size_t)s->t * ny * nx;                      \
    for (int y = lo; y < hi; ++y)                                                      \
      for (int x = 0; x < nx; ++x) {                                                   \
        hx[IDX(s->tfsf_z, y, x)] += Db * iey[(size_t)y * nx + x];                      \
        hy[IDX(s->tfsf_z, y, x)] -= Db * iex[(size_t)y * nx + x];                      \
      }                                                                                \
  }                                                                                    \
  /* ---- phase 3: E main update, per row as phase 0 ---- */                     \
  if (phase == 3)                                                                      \
  for (int z = lo; z < hi && z < nz - 1; ++z)                                          \
    for (int y = 0; y < ny - 1; ++y) {                                                 \
      const size_t r = IDX(z, y, 0);                                                   \
      T *RS exr = ex + r; T *RS eyr = ey + r; T *RS ezr = ez + r;                      \
      const T *RS car = ca + r; const T *RS cbr = cb + r;                              \
      const T *RS hxr = hx + r; const T *RS hyr = hy + r; const T *RS hzr = hz + r;    \
      if (z >= 1) {                                                                    \
        const T *RS hyz = hy + IDX(z - 1, y, 0); const T *RS hxz = hx + IDX(z - 1, y, 0); \
        if (y >= 1) {                                                                  \
          const T *RS hzy = hz + IDX(z, y - 1, 0);                                     \
          for (int x = 0; x < nx - 1; ++x)                                             \
            exr[x] = (exr[x] * car[x]) + (cbr[x] * ((hzr[x] - hzy[x]) - (hyr[x] - hyz[x]))); \
        }                                                                              \
        for (int x = 1; x < nx - 1; ++x)                                               \
          eyr[x] = (eyr[x] * car[x]) + (cbr[x] * ((hxr[x] - hxz[x]) - (hzr[x] - hzr[x - 1]))); \
      }                                                                                \
      if (y >= 1) {                                                                    \
        const T *RS hxy = hx + IDX(z, y - 1, 0);                                       \
        for (int x = 1; x < nx - 1; ++x)                                               \
          ezr[x] = (ezr[x] * car[x]) + (cbr[x] * ((hyr[x] - hyr[x - 1]) - (hxr[x] - hxy[x]))); \
      }                                                                                \
    }                                                                                  \
  /* ---- phase 4: E CPML over the face regions: z faces, then x, then y ---- */      \
  /* phase 8: E z faces, rows of the face planes [lo, hi) (planes            \
   * 1 <= z < m and nz - m <= z < nz - 1); then phase 4: x and y faces */        \
  if (phase == 8)                                                                      \
  for (int w = lo; w < hi; ++w) {                                                      \
    const int j = w / (ny - 1), y = w % (ny - 1);                                      \
    const int sd = j < m - 1 ? 0 : 1, q = sd ? j - (m - 1) : j + 1;                    \
    const int z = sd ? nz - m + q : q;                                                 \
    const T b = be[sd][q], c = cE[sd][q];                                              \
    const size_t r = IDX(z, y, 0), rz = IDX(z - 1, y, 0);                              \
    T *RS Pyz = (T *)s->psi[0][sd][1] + ((size_t)q * ny + y) * nx;                     \
    T *RS Pxz = (T *)s->psi[0][sd][0] + ((size_t)q * ny + y) * nx;                     \
    T *RS exr = ex + r; T *RS eyr = ey + r;                                            \
    const T *RS cbr = cb + r;                                                          \
    const T *RS hxr = hx + r; const T *RS hyr = hy + r;                                \
    const T *RS hxz = hx + rz; const T *RS hyz = hy + rz;                              \
    for (int x = 0; x < nx - 1; ++x) {                                                 \
      Pyz[x] = b * Pyz[x] + c * (hxr[x] - hxz[x]) / dx;                                \
      Pxz[x] = b * Pxz[x] + c * (hyr[x] - hyz[x]) / dx;                                \
      eyr[x] += cbr[x] * dx * Pyz[x];                                                  \
      exr[x] -= cbr[x] * dx * Pxz[x];                                                  \
    }                                                                                  \
  }                                                                                    \
  if (phase == 4)                                                                      \
  for (int z = lo; z < hi && z < nz - 1; ++z) {                                        \
    for (int y = 0; y < ny - 1; ++y)                                                   \
      for (int sx = 0; sx < 2; ++sx) {                                                 \
        const int x0 = sx ? nx - m : 1, x1 = sx ? nx - 1 : m;                          \
        for (int x = x0; x < x1; ++x) {                                                \
          const int qx = sx ? x - (nx - m) : x;                                        \
          const size_t i = IDX(z, y, x);                                               \
          T *Pzx = (T *)s->psi[1][sx][1], *Pyx = (T *)s->psi[1][sx][0];                \
          const size_t k = ((size_t)z * ny + y) * m + qx;                              \
          const T b = be[sx][qx], c = cE[sx][qx];                                      \
          Pzx[k] = b * Pzx[k] + c * (hy[i] - hy[i - 1]) / dx;                          \
          Pyx[k] = b * Pyx[k] + c * (hz[i] - hz[i - 1]) / dx;                          \
          ez[i] += cb[i] * dx * Pzx[k];                                                \
          ey[i] -= cb[i] * dx * Pyx[k];                                                \
        }                                                                              \
      }                                                                                \
    for (int sy = 0; sy < 2; ++sy) {                                                   \
      const int y0 = sy ? ny - m : 1, y1 = sy ? ny - 1 : m;                            \
      for (int y = y0; y < y1; ++y) {                                                  \
        const int qy = sy ? y - (ny - m) : y;                                          \
        const T b = be[sy][qy], c = cE[sy][qy];                                        \
        const size_t r = IDX(z, y, 0), ry = IDX(z, y - 1, 0);                          \
        T *RS Pxy = (T *)s->psi[2][sy][0] + ((size_t)z * m + qy) * nx;                 \
        T *RS Pzy = (T *)s->psi[2][sy][1] + ((size_t)z * m + qy) * nx;                 \
        T *RS exr = ex + r; T *RS ezr = ez + r;                                        \
        const T *RS cbr = cb + r;                                                      \
        const T *RS hxr = hx + r; const T *RS hzr = hz + r;                            \
        const T *RS hxy = hx + ry; const T *RS hzy = hz + ry;                          \
        for (int x = 0; x < nx - 1; ++x) {                                             \
          Pxy[x] = b * Pxy[x] + c * (hzr[x] - hzy[x]) / dx;                            \
          Pzy[x] = b * Pzy[x] + c * (hxr[x] - hxy[x]) / dx;                            \
          exr[x] += cbr[x] * dx * Pxy[x];                                              \
          ezr[x] -= cbr[x] * dx * Pzy[x];                                              \
        }                                                                              \
      }                                                                                \
    }                                                                                  \
  }                                                                                    \
  /* ---- phase 5: H-field injection into E ---- */                                   \
  if (phase == 5 && inj) {                                                             \
    const T *ihx = (const T *)s->inc[2] + (size_t)s->t * ny * nx;                      \
    const T *ihy = (const T *)s->inc[3] + (size_t)s->t * ny * nx;                      \
    for (int y = lo; y < hi; ++y)                                                      \
      for (int x = 0; x < nx; ++x) {                                                   \
        ey[IDX(s->tfsf_z, y, x)] += dte0dx * ihx[(size_t)y * nx + x];                  \
        ex[IDX(s->tfsf_z, y, x)] -= dte0dx * ihy[(size_t)y * nx + x];                  \
      }                                                                                \
  }                                                                                    \
  /* ---- phase 6: phasors, plane groups [lo, hi) ---- */                             \
  const int nxp = nx - 2 * m, nyp = ny - 2 * m, nzp = nz - 2 * m;                      \
  const double cEp = s->ce, sEp = s->se, cHp = s->ch, sHp = s->sh;                     \
  if (phase == 6)                                                                      \
  for (int g = lo; g < hi; ++g) {                                                      \
    const int d0 = g < 2 ? nyp : nzp, d1 = g < 2 ? nxp : (g < 4 ? nyp : nxp);          \
    for (int a = 1; a < d0; ++a)                                                       \
      for (int b = 1; b < d1; ++b) {                                                   \
        const size_t k = (size_t)a * d1 + b;                                           \
        double mv[4];                                                                  \
        int base;                                                                      \
        if (g < 2) {                                                                   \
          const int pz = g == 0 ? m + 1 : nz - m - 1, yy = m + a, xx = m + b;          \
          base = g * 4;                                                                \
          mv[0] = 0.5 * (double)(T)(ex[IDX(pz, yy, xx)] + ex[IDX(pz, yy, xx - 1)]);    \
          mv[1] = 0.5 * (double)(T)(ey[IDX(pz, yy, xx)] + ey[IDX(pz, yy - 1, xx)]);    \
          mv[2] = 0.25 * (double)(T)(hx[IDX(pz, yy, xx)] + hx[IDX(pz, yy - 1, xx)] +   \
                                     hx[IDX(pz - 1, yy, xx)] + hx[IDX(pz - 1, yy - 1, xx)]); \
          mv[3] = 0.25 * (double)(T)(hy[IDX(pz, yy, xx)] + hy[IDX(pz, yy, xx - 1)] +   \
                                     hy[IDX(pz - 1, yy, xx)] + hy[IDX(pz - 1, yy, xx - 1)]); \
        } else if (g < 4) {                                                            \
          const int px = g == 2 ? m + 1 : nx - m - 1, zz = m + a, yy = m + b;          \
          base = 8 + (g - 2) * 4;                                                      \
          mv[0] = 0.5 * (double)(T)(ey[IDX(zz, yy, px)] + ey[IDX(zz, yy - 1, px)]);    \
          mv[1] = 0.5 * (double)(T)(ez[IDX(zz, yy, px)] + ez[IDX(zz - 1, yy, px)]);    \
          mv[2] = 0.25 * (double)(T)(hy[IDX(zz, yy, px)] + hy[IDX(zz, yy, px - 1)] +   \
                                     hy[IDX(zz - 1, yy, px)] + hy[IDX(zz - 1, yy, px - 1)]); \
          mv[3] = 0.25 * (double)(T)(hz[IDX(zz, yy, px)] + hz[IDX(zz, yy, px - 1)] +   \
                                     hz[IDX(zz, yy - 1, px)] + hz[IDX(zz, yy - 1, px - 1)]); \
        } else {                                                                       \
          const int py = g == 4 ? m + 1 : ny - m - 1, zz = m + a, xx = m + b;          \
          base = 16 + (g - 4) * 4;                                                     \
          mv[0] = 0.5 * (double)(T)(ex[IDX(zz, py, xx)] + ex[IDX(zz, py, xx - 1)]);    \
          mv[1] = 0.5 * (double)(T)(ez[IDX(zz, py, xx)] + ez[IDX(zz - 1, py, xx)]);    \
          mv[2] = 0.25 * (double)(T)(hx[IDX(zz, py, xx)] + hx[IDX(zz, py - 1, xx)] +   \
                                     hx[IDX(zz - 1, py, xx)] + hx[IDX(zz - 1, py - 1, xx)]); \
          mv[3] = 0.25 * (double)(T)(hz[IDX(zz, py, xx)] + hz[IDX(zz, py - 1, xx)] +   \
                                     hz[IDX(zz, py, xx - 1)] + hz[IDX(zz, py - 1, xx - 1)]); \
        }                                                                              \
        for (int c = 0; c < 4; ++c) {                                                  \
          T *p = (T *)s->ph[base + c] + 2 * k;                                         \
          const double cc = c < 2 ? cEp : cHp, ss = c < 2 ? sEp : sHp;                 \
          p[0] = (T)((double)p[0] + mv[c] * cc);                                       \
          p[1] = (T)((double)p[1] + mv[c] * ss);                                       \
        }                                                                              \
      }                                                                                \
  }                                                                                    \
}

DEFINE_STEP(float, phase_f32)
DEFINE_STEP(double, phase_f64)

typedef struct job {
  const oracle_state *s;
  int phase, lo, hi;
} job;

static void *run_job(void *arg) {
  const job *j = (const job *)arg;
  if (j->s->dtype == 0) phase_f32(j->s, j->phase, j->lo, j->hi);
  else phase_f64(j->s, j->phase, j->lo, j->hi);
  return NULL;
}

/* Runs one phase over [0, n) split into contiguous ranges, one per thread
 * (each range writes only its own cells). */
static int run_phase(const oracle_state *s, int phase, int n) {
  enum { kMaxThreads = 256 };
  int nt = s->nthreads < 1 ? 1 : (s->nthreads > kMaxThreads ? kMaxThreads : s->nthreads);
  if (nt > n) nt = n < 1 ? 1 : n;
  job jobs[kMaxThreads];
  pthread_t th[kMaxThreads];
  for (int k = 0; k < nt; ++k) {
    jobs[k].s = s;
    jobs[k].phase = phase;
    jobs[k].lo = (int)((long long)n * k / nt);
    jobs[k].hi = (int)((long long)n * (k + 1) / nt);
  }
  int started = 0;
  for (int k = 1; k < nt; ++k) {
    if (pthread_create(&th[k], NULL, run_job, &jobs[k]) != 0) break;
    started = k;
  }
  run_job(&jobs[0]);
  for (int k = started + 1; k < nt; ++k) run_job(&jobs[k]);   /* threads that did not start */
  for (int k = 1; k <= started; ++k) pthread_join(th[k], NULL);
  return 0;
}

/* One time step of the state. Returns 0, or 1 for a bad element type. */
int oracle_step(const oracle_state *s) {
  if (s->dtype != 0 && s->dtype != 1) return 1;
  const int zrows = (s->npml - 1) * 2 * (s->ny - 1);   /* z-face rows of either kind */
  run_phase(s, 0, s->nz);   /* H main */
  run_phase(s, 7, zrows);   /* H CPML, z faces */
  run_phase(s, 1, s->nz);   /* H CPML, x and y faces */
  run_phase(s, 2, s->ny);   /* injection into H */
  run_phase(s, 3, s->nz);   /* E main */
  run_phase(s, 8, zrows);   /* E CPML, z faces */
  run_phase(s, 4, s->nz);   /* E CPML, x and y faces */
  run_phase(s, 5, s->ny);   /* injection into E */
  run_phase(s, 6, 6);       /* phasors */
  return 0;
}
