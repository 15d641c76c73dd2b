/* On-device image driver: the base image and the adaptive-refinement levels
 * of ipole's fast-light loop (src/main.c:520-792), with save_pixel
 * (:885-910), save_pixelTransfer/lininterp2/lininterp4 (:912-999) and the
 * flux estimate that scales the absolute criterion (:597-626).
 *
 * The image stays in device memory from the first level to the last; each
 * level's pixel list is built, compacted and traced on the device.  Per level
 * the host reads back one small status record (the list length and the
 * error and oddity counters) and, only when a ray reported an oddity, the
 * traced list for the log.
 *
 * Why a level is data-parallel: a pixel of level l (spacing ns) lies on an
 * odd multiple of ns in i or j, and every value its criterion and its
 * interpolation read lies on even multiples of ns in both (the corners and
 * edge mid-points of the coarser grid), which earlier levels wrote.  So all
 * candidates of a level are independent, and their order matters only for
 * the traced list, which an order-preserving scan keeps in the reference's
 * row-major loop order (the order of its oddity and MaxNStep messages).
 *
 * Arithmetic: the criteria, the averages and the flux estimate are the host
 * driver's expressions in the same order (no multiply-add pairs to contract),
 * and the flux estimate is summed in the reference's index order by a single
 * thread, so the image is bit-identical to the host driver's. */
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "ipg_internal.h"
#include "ipole_b200.h"
#include "ipole_host.h"

#define NIMG 5
#define TPB 256
#define SCAN_TPB 1024

struct RefineStatus {
  int n;            /* pixels to trace at this level (compaction total) */
  int interpolated; /* interpolated pixels in the image (interp_flag set) */
  int nan;          /* a NaN was met in save_pixel or an interpolation */
  int maxn_first;   /* first list position whose ray hit maxnstep, INT_MAX if none */
  int odd;          /* traced rays with an oddity to report */
  int pad;
  double Iavg;      /* flux estimate per pixel (main.c:620-626) */
};

struct RefineBufs {
  size_t cap;  /* pixels */
  size_t cap_prelim;
  double *image, *taus, *imageS;
  int32_t *interp, *oddflag, *nstep;
  int32_t *ij, *flags, *block_sums;
  ipg_pixel_out *out;
  double *prelim;
  int32_t *winner;
  RefineStatus *st;
  RefineStatus *h_st; /* pinned */
};

extern "C" void ipg__refine_release(void *p)
{
  RefineBufs *r = (RefineBufs *)p;
  if (!r) return;
  cudaFree(r->image);
  cudaFree(r->taus);
  cudaFree(r->imageS);
  cudaFree(r->interp);
  cudaFree(r->oddflag);
  cudaFree(r->nstep);
  cudaFree(r->ij);
  cudaFree(r->flags);
  cudaFree(r->block_sums);
  cudaFree(r->out);
  cudaFree(r->prelim);
  cudaFree(r->winner);
  cudaFree(r->st);
  cudaFreeHost(r->h_st);
  free(r);
}

/* ---------------------------------------------------------------- kernels */

/* base-image pixel list in the loop order of main.c:536-537 */
__global__ void k_base_list(int32_t *ij, int ni, int nj, int sx, int sy)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ni * nj) return;
  ij[2 * t] = (t / nj) * sx;
  ij[2 * t + 1] = (t % nj) * sy;
}

/* MaxNStep (first list position) and oddity count of a traced list: the
 * checks of ipg_trace_pixels and get_pixel (main.c:841-869) */
__global__ void k_check(const ipg_pixel_out *out, int n, int maxnstep, int unpol, RefineStatus *st)
{
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  ipg_pixel_out o = out[m];
  if (o.nstep >= maxnstep - 1) atomicMin(&st->maxn_first, m);
  if (o.flag != 0 || (!unpol && o.I < -1.e-10)) atomicAdd(&st->odd, 1);
}

struct ImgPtrs {
  double *image, *taus, *imageS;
  int32_t *interp, *oddflag, *nstep;
  int ny;
};

/* save_pixel (main.c:885-910) for every traced pixel; interp_flag = 0 */
__global__ void k_save(const int32_t *ij, const ipg_pixel_out *out, int n, ImgPtrs P, double f3, int unpol,
                       int qu_conv, RefineStatus *st)
{
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  size_t p = (size_t)ij[2 * m] * P.ny + ij[2 * m + 1];
  ipg_pixel_out o = out[m];
  P.image[p] = o.I_unpol * f3;
  P.taus[p] = o.tau;
  P.oddflag[p] = o.flag;
  P.nstep[p] = o.nstep;
  P.interp[p] = 0;
  if (!unpol) {
    double *s = P.imageS + p * NIMG;
    s[0] = o.I * f3;
    if (qu_conv == 0) {
      s[1] = -o.Q * f3;
      s[2] = -o.U * f3;
    } else {
      s[1] = o.Q * f3;
      s[2] = o.U * f3;
    }
    s[3] = o.V * f3;
    s[4] = o.tauF;
    if (isnan(s[0])) atomicOr(&st->nan, 1);
  }
}

/* prelim location and weight of one base pixel (main.c:597-613); the
 * location expression mixes sx and sy exactly as the reference does */
__device__ __forceinline__ void prelim_of(int i, int j, int nx, int ny, int nymin, int sx, int sy, double I,
                                          long long *loc, double *v)
{
  *loc = (long long)(i / sy) * nymin + j / sx;
  const double dsx = (double)sx;
  if (i % (nx - 1) != 0 && j % (ny - 1) != 0) *v = I * dsx * dsx;
  else if ((i == 0 && j % (ny - 1) != 0) || (i % (nx - 1) != 0 && j == 0)) *v = I * (double)(sx / 2 + 1) * dsx;
  else if (i % (nx - 1) != 0 || j % (ny - 1) != 0) *v = I * (double)(sx / 2) * dsx;
  else if (i == 0 && j == 0) *v = I * (double)(sx / 2 + 1) * (double)(sx / 2 + 1);
  else if (i == 0 || j == 0) *v = I * (double)(sx / 2 + 1) * dsx / 2;
  else *v = I * (double)(sx * sx) / 4;
}

/* the last base pixel (in list order) that writes each prelim slot wins, as
 * in the reference's sequential loop */
__global__ void k_prelim_claim(const int32_t *ij, int n, int nx, int ny, int nymin, int sx, int sy, long long nslot,
                               int32_t *winner)
{
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  long long loc;
  double v;
  prelim_of(ij[2 * q], ij[2 * q + 1], nx, ny, nymin, sx, sy, 0., &loc, &v);
  if (loc >= 0 && loc < nslot) atomicMax(&winner[loc], q);
}

__global__ void k_prelim_fill(const int32_t *ij, const ipg_pixel_out *out, int n, int nx, int ny, int nymin, int sx,
                              int sy, long long nslot, const int32_t *winner, double *prelim)
{
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  long long loc;
  double v;
  prelim_of(ij[2 * q], ij[2 * q + 1], nx, ny, nymin, sx, sy, out[q].I_unpol, &loc, &v);
  if (loc >= 0 && loc < nslot && winner[loc] == q) prelim[loc] = v;
}

/* interp_tot summed in index order by one thread (the reference's order, so
 * the same rounding); the warp stages the values through shared memory */
__global__ void k_prelim_sum(const double *prelim, long long nslot, double f3, double npix, RefineStatus *st)
{
  __shared__ double buf[1024];
  double tot = 0.;
  for (long long base = 0; base < nslot; base += 1024) {
    long long m = nslot - base < 1024 ? nslot - base : 1024;
    for (long long k = threadIdx.x; k < m; k += blockDim.x) buf[k] = prelim[base + k];
    __syncwarp();
    if (threadIdx.x == 0)
      for (long long k = 0; k < m; k++) tot += buf[k];
    __syncwarp();
  }
  if (threadIdx.x == 0) st->Iavg = tot * f3 / npix;
}

struct LevelArgs {
  int nx, ny, nsx, nsy, psx, psy, ni, nj;
  int unpol, nearest;
  double refine_abs, refine_rel, refine_cut;
};

__device__ __forceinline__ bool avg2(ImgPtrs P, int unpol, size_t a, size_t b, size_t d)
{
  P.image[d] = .5 * (P.image[a] + P.image[b]);
  P.taus[d] = .5 * (P.taus[a] + P.taus[b]);
  if (unpol) return false;
  for (int c = 0; c < NIMG; c++) P.imageS[d * NIMG + c] = .5 * (P.imageS[a * NIMG + c] + P.imageS[b * NIMG + c]);
  return isnan(P.imageS[a * NIMG]) || isnan(P.imageS[b * NIMG]);
}

__device__ __forceinline__ bool avg4(ImgPtrs P, int unpol, size_t a, size_t b, size_t c3, size_t e, size_t d)
{
  P.image[d] = .25 * (P.image[a] + P.image[b] + P.image[c3] + P.image[e]);
  P.taus[d] = .25 * (P.taus[a] + P.taus[b] + P.taus[c3] + P.taus[e]);
  if (unpol) return false;
  for (int c = 0; c < NIMG; c++)
    P.imageS[d * NIMG + c] = .25 * (P.imageS[a * NIMG + c] + P.imageS[b * NIMG + c] + P.imageS[c3 * NIMG + c] +
                                    P.imageS[e * NIMG + c]);
  return isnan(P.imageS[a * NIMG]) || isnan(P.imageS[b * NIMG]) || isnan(P.imageS[c3 * NIMG]) ||
         isnan(P.imageS[e * NIMG]);
}

__device__ __forceinline__ bool copy1(ImgPtrs P, int unpol, size_t a, size_t d)
{
  P.image[d] = P.image[a];
  if (unpol) return false;
  P.taus[d] = P.taus[a];
  for (int c = 0; c < NIMG; c++) P.imageS[d * NIMG + c] = P.imageS[a * NIMG + c];
  return isnan(P.imageS[a * NIMG]);
}

/* one refinement level (main.c:640-777): criterion per candidate pixel;
 * flags[t] = 1 marks a pixel to trace, the others are interpolated here */
__global__ void k_level(LevelArgs L, ImgPtrs P, const RefineStatus *stin, int32_t *flags, RefineStatus *st)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < L.ni * L.nj) {
    const int i = (t / L.nj) * L.nsx, j = (t % L.nj) * L.nsy;
    int flag = 0;
    if (!(i % L.psx == 0 && j % L.psy == 0)) {
      const double Iavg = stin->Iavg;
      const size_t ny = (size_t)L.ny;
      /* the +ns neighbours exist unless the spacing does not divide the
       * image (a base-to-final ratio that is not a power of two), where the
       * reference reads past the image: such a pixel is traced */
      const bool inside = (i % L.psx == 0 || i + L.nsx <= L.nx - 1) && (j % L.psy == 0 || j + L.nsy <= L.ny - 1);
      double I1 = 0., I2 = 0., I3 = 0., err_abs = 0., err_rel = 0.;
      if (!inside) {
      } else if (i % L.psx == 0) {
        I1 = P.image[i * ny + j - L.nsy];
        I2 = P.image[i * ny + j + L.nsy];
        err_abs = (I2 - I1) / 2 / Iavg;
        err_rel = (I2 - I1) / 2 / I1;
      } else if (j % L.psy == 0) {
        I1 = P.image[(i - L.nsx) * ny + j];
        I2 = P.image[(i + L.nsx) * ny + j];
        err_abs = (I2 - I1) / 2 / Iavg;
        err_rel = (I2 - I1) / 2 / I1;
      } else {
        I1 = P.image[(i - L.nsx) * ny + j - L.nsy];
        I2 = P.image[(i + L.nsx) * ny + j - L.nsy];
        I3 = P.image[(i - L.nsx) * ny + j + L.nsy];
        err_abs = ((I2 + I3) / 2 - I1) / Iavg;
        err_rel = (I2 + I3) / (2 * I1) - 1.;
      }
      const size_t d = (size_t)i * ny + j;
      if (!inside || ((fabs(err_abs) > L.refine_abs && fabs(err_rel) > L.refine_rel) && fabs(I1) > L.refine_cut)) {
        flag = 1;
        P.interp[d] = 0;
      } else {
        P.interp[d] = 1;
        bool bad;
        if (i % L.psx == 0) {
          bad = L.nearest ? copy1(P, L.unpol, d - L.nsy, d) : avg2(P, L.unpol, d - L.nsy, d + L.nsy, d);
        } else if (j % L.psy == 0) {
          bad = L.nearest ? copy1(P, L.unpol, d - L.nsx * ny, d)
                          : avg2(P, L.unpol, d - L.nsx * ny, d + L.nsx * ny, d);
        } else {
          bad = L.nearest ? copy1(P, L.unpol, d - L.nsx * ny - L.nsy, d)
                          : avg4(P, L.unpol, d - L.nsx * ny - L.nsy, d + L.nsx * ny - L.nsy,
                                 d - L.nsx * ny + L.nsy, d + L.nsx * ny + L.nsy, d);
        }
        if (bad) atomicOr(&st->nan, 1);
      }
    }
    flags[t] = flag;
  }
}

/* number of interpolated pixels in the whole image (main.c:781-783) */
__global__ void k_count_interp(const int32_t *interp, int npix, RefineStatus *st)
{
  int c = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) c += interp[p] != 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&st->interpolated, c);
}

/* order-preserving compaction of the flagged candidates: per-block counts,
 * one block scanning the block counts, then the scatter */
__device__ __forceinline__ int block_exclusive_scan(int v, int *total)
{
  __shared__ int warp_sums[SCAN_TPB / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sums[lane] = s;
  }
  __syncthreads();
  int excl = x - v + (w > 0 ? warp_sums[w - 1] : 0);
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(SCAN_TPB) k_scan_blocks(const int32_t *flags, int n, int32_t *block_sums)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int tot;
  block_exclusive_scan(t < n ? flags[t] : 0, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_TPB) k_scan_top(int32_t *block_sums, int nb, RefineStatus *st)
{
  int carry = 0;
  for (int base = 0; base < nb; base += SCAN_TPB) {
    int k = base + threadIdx.x;
    int v = k < nb ? block_sums[k] : 0, tot;
    int e = block_exclusive_scan(v, &tot);
    if (k < nb) block_sums[k] = carry + e;
    carry += tot;
  }
  if (threadIdx.x == 0) st->n = carry;
}

__global__ void __launch_bounds__(SCAN_TPB) k_scatter(const int32_t *flags, int n, const int32_t *block_sums,
                                                      int nj, int nsx, int nsy, int32_t *ij)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int f = t < n ? flags[t] : 0;
  int e = block_exclusive_scan(f, NULL);
  if (f) {
    int pos = block_sums[blockIdx.x] + e;
    ij[2 * pos] = (t / nj) * nsx;
    ij[2 * pos + 1] = (t % nj) * nsy;
  }
}

/* ------------------------------------------------------------------ host */

#define CKR(call)                                                                            \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      char m_[400];                                                                          \
      snprintf(m_, sizeof(m_), "%s: %s", #call, cudaGetErrorString(e_));                     \
      ipg__set_error(ctx, m_);                                                               \
      return IPG_E_CUDA;                                                                     \
    }                                                                                        \
  } while (0)

static int grid_of(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

static int ensure_bufs(ipg_ctx *ctx, size_t npix, size_t nprelim, RefineBufs **out)
{
  RefineBufs **slot = (RefineBufs **)ipg__refine_slot(ctx);
  RefineBufs *r = *slot;
  if (!r) {
    r = (RefineBufs *)calloc(1, sizeof(RefineBufs));
    if (!r) return IPG_E_NOMEM;
    *slot = r;
    CKR(cudaMalloc(&r->st, sizeof(RefineStatus)));
    CKR(cudaMallocHost(&r->h_st, sizeof(RefineStatus)));
  }
  if (r->cap < npix) {
    cudaFree(r->image);
    cudaFree(r->taus);
    cudaFree(r->imageS);
    cudaFree(r->interp);
    cudaFree(r->oddflag);
    cudaFree(r->nstep);
    cudaFree(r->ij);
    cudaFree(r->flags);
    cudaFree(r->block_sums);
    cudaFree(r->out);
    r->cap = 0;
    CKR(cudaMalloc(&r->image, npix * sizeof(double)));
    CKR(cudaMalloc(&r->taus, npix * sizeof(double)));
    CKR(cudaMalloc(&r->imageS, npix * NIMG * sizeof(double)));
    CKR(cudaMalloc(&r->interp, npix * sizeof(int32_t)));
    CKR(cudaMalloc(&r->oddflag, npix * sizeof(int32_t)));
    CKR(cudaMalloc(&r->nstep, npix * sizeof(int32_t)));
    CKR(cudaMalloc(&r->ij, 2 * npix * sizeof(int32_t)));
    CKR(cudaMalloc(&r->flags, npix * sizeof(int32_t)));
    CKR(cudaMalloc(&r->block_sums, (npix / SCAN_TPB + 2) * sizeof(int32_t)));
    CKR(cudaMalloc(&r->out, npix * sizeof(ipg_pixel_out)));
    r->cap = npix;
  }
  if (r->cap_prelim < nprelim) {
    cudaFree(r->prelim);
    cudaFree(r->winner);
    r->cap_prelim = 0;
    CKR(cudaMalloc(&r->prelim, nprelim * sizeof(double)));
    CKR(cudaMalloc(&r->winner, nprelim * sizeof(int32_t)));
    r->cap_prelim = nprelim;
  }
  *out = r;
  return IPG_OK;
}

static int reset_status(ipg_ctx *ctx, RefineBufs *r, cudaStream_t s)
{
  RefineStatus z;
  memset(&z, 0, sizeof(z));
  z.maxn_first = INT_MAX;
  /* keep Iavg: the levels read it */
  CKR(cudaMemcpyAsync(r->st, &z, offsetof(RefineStatus, Iavg), cudaMemcpyHostToDevice, s));
  return IPG_OK;
}

static int read_status(ipg_ctx *ctx, RefineBufs *r, cudaStream_t s)
{
  CKR(cudaMemcpyAsync(r->h_st, r->st, sizeof(RefineStatus), cudaMemcpyDeviceToHost, s));
  CKR(cudaStreamSynchronize(s));
  return IPG_OK;
}

/* trace r->ij[0..n) into r->out and apply get_pixel's checks and logs */
static int trace_level(ipg_ctx *ctx, const ipg_camera *cam, const ipg_refine_args *a, RefineBufs *r, size_t n,
                       ImgPtrs P, FILE *log)
{
  cudaStream_t s = (cudaStream_t)ipg__stream(ctx);
  int rc = ipg__trace_core(ctx, cam, r->ij, n, r->out);
  if (rc != IPG_OK) {
    if (log) fprintf(log, "trace failed: %s\n", ipg_strerror(rc));
    return rc;
  }
  if ((rc = reset_status(ctx, r, s))) return rc;
  k_check<<<grid_of((long long)n, TPB), TPB, 0, s>>>(r->out, (int)n, cam->maxnstep, a->only_unpolarized, r->st);
  CKR(cudaGetLastError());
  if ((rc = read_status(ctx, r, s))) return rc;
  if (r->h_st->maxn_first != INT_MAX) {
    int32_t pij[2];
    CKR(cudaMemcpy(pij, r->ij + 2 * (size_t)r->h_st->maxn_first, sizeof(pij), cudaMemcpyDeviceToHost));
    if (log) fprintf(log, "\nMaxNStep exceeded in pixel %d %d!\n", pij[0], pij[1]);
    char m[128];
    snprintf(m, sizeof(m), "MaxNStep exceeded in pixel %d %d", pij[0], pij[1]);
    ipg__set_error(ctx, m);
    return IPG_E_MAXNSTEP;
  }
  if (r->h_st->odd && log) {
    std::vector<int32_t> hij(2 * n);
    std::vector<ipg_pixel_out> hout(n);
    CKR(cudaMemcpy(hij.data(), r->ij, 2 * n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    CKR(cudaMemcpy(hout.data(), r->out, n * sizeof(ipg_pixel_out), cudaMemcpyDeviceToHost));
    ipg__report_oddities(a->only_unpolarized, hij.data(), hout.data(), n, log);
  }
  k_save<<<grid_of((long long)n, TPB), TPB, 0, s>>>(r->ij, r->out, (int)n, P, a->f3, a->only_unpolarized,
                                                      a->qu_conv, r->st);
  CKR(cudaGetLastError());
  if ((rc = read_status(ctx, r, s))) return rc;
  if (r->h_st->nan) {
    fprintf(stderr, "NaN in image! Exiting.\n");
    return IPG_E_NAN;
  }
  return IPG_OK;
}

extern "C" int ipg__render_levels_device(ipg_ctx *ctx, const ipg_camera *cam, const ipg_refine_args *a, void *imgp,
                                         FILE *log)
{
  ipg_image *img = (ipg_image *)imgp;
  const size_t nx = a->nx, ny = a->ny, npix = nx * ny;
  if (npix >= (size_t)INT_MAX / 2 || a->nxmin < 2 || a->nymin < 2) return IPG_E_ARG;
  const size_t nprelim = a->refine_level > 1 ? a->nxmin * a->nymin : 1;
  RefineBufs *r;
  int rc = ensure_bufs(ctx, npix, nprelim, &r);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)ipg__stream(ctx);
  ImgPtrs P = {r->image, r->taus, r->imageS, r->interp, r->oddflag, r->nstep, (int)ny};
  CKR(cudaMemsetAsync(r->image, 0, npix * sizeof(double), s));
  CKR(cudaMemsetAsync(r->taus, 0, npix * sizeof(double), s));
  if (!a->only_unpolarized) CKR(cudaMemsetAsync(r->imageS, 0, npix * NIMG * sizeof(double), s));
  CKR(cudaMemsetAsync(r->interp, 0, npix * sizeof(int32_t), s));
  CKR(cudaMemsetAsync(r->oddflag, 0, npix * sizeof(int32_t), s));
  CKR(cudaMemsetAsync(r->nstep, 0, npix * sizeof(int32_t), s));
  {
    RefineStatus z;
    memset(&z, 0, sizeof(z));
    z.maxn_first = INT_MAX;
    CKR(cudaMemcpyAsync(r->st, &z, sizeof(z), cudaMemcpyHostToDevice, s));
  }

  /* base image, main.c:535-615 */
  const int sx = (int)((nx - 1) / (a->nxmin - 1)), sy = (int)((ny - 1) / (a->nymin - 1));
  const int ni = (int)((nx - 1) / sx + 1), nj = (int)((ny - 1) / sy + 1);
  size_t n = (size_t)ni * nj;
  k_base_list<<<grid_of((long long)n, TPB), TPB, 0, s>>>(r->ij, ni, nj, sx, sy);
  CKR(cudaGetLastError());
  if ((rc = trace_level(ctx, cam, a, r, n, P, log))) return rc;
  size_t traced = n;

  if (a->refine_level > 1) {
    const long long nslot = (long long)nprelim;
    CKR(cudaMemsetAsync(r->prelim, 0, nprelim * sizeof(double), s));
    CKR(cudaMemsetAsync(r->winner, 0xff, nprelim * sizeof(int32_t), s));
    k_prelim_claim<<<grid_of((long long)n, TPB), TPB, 0, s>>>(r->ij, (int)n, (int)nx, (int)ny, (int)a->nymin, sx,
                                                               sy, nslot, r->winner);
    k_prelim_fill<<<grid_of((long long)n, TPB), TPB, 0, s>>>(r->ij, r->out, (int)n, (int)nx, (int)ny,
                                                              (int)a->nymin, sx, sy, nslot, r->winner, r->prelim);
    k_prelim_sum<<<1, 32, 0, s>>>(r->prelim, nslot, a->f3, (double)npix, r->st);
    CKR(cudaGetLastError());
  }

  /* refinement levels, main.c:635-792 */
  for (int lvl = 1; lvl < a->refine_level; lvl++) {
    LevelArgs L;
    L.nx = (int)nx;
    L.ny = (int)ny;
    L.nsx = (int)(sx / pow(2, lvl));
    L.nsy = (int)(sy / pow(2, lvl));
    L.psx = 2 * L.nsx;
    L.psy = 2 * L.nsy;
    if (L.nsx < 1 || L.nsy < 1) { /* the reference loops forever here */
      if (log) fprintf(log, "refinement spacing below one pixel at level %d: nx_min/ny_min too small\n", lvl + 1);
      return IPG_E_ARG;
    }
    L.ni = (int)((nx - 1) / L.nsx + 1);
    L.nj = (int)((ny - 1) / L.nsy + 1);
    L.unpol = a->only_unpolarized;
    L.nearest = a->nearest_neighbor;
    L.refine_abs = a->refine_abs;
    L.refine_rel = a->refine_rel;
    L.refine_cut = a->refine_cut;
    if (log) fprintf(log, "Refining level %d of %d, spacing %d,%d\n", lvl + 1, a->refine_level, L.nsx, L.nsy);
    if ((rc = reset_status(ctx, r, s))) return rc;
    const int ncand = L.ni * L.nj, nb = grid_of(ncand, SCAN_TPB);
    k_level<<<grid_of(ncand, TPB), TPB, 0, s>>>(L, P, r->st, r->flags, r->st);
    k_scan_blocks<<<nb, SCAN_TPB, 0, s>>>(r->flags, ncand, r->block_sums);
    k_scan_top<<<1, SCAN_TPB, 0, s>>>(r->block_sums, nb, r->st);
    k_scatter<<<nb, SCAN_TPB, 0, s>>>(r->flags, ncand, r->block_sums, L.nj, L.nsx, L.nsy, r->ij);
    k_count_interp<<<grid_of((long long)npix, TPB) < 1184 ? grid_of((long long)npix, TPB) : 1184, TPB, 0, s>>>(
        r->interp, (int)npix, r->st);
    CKR(cudaGetLastError());
    if ((rc = read_status(ctx, r, s))) return rc;
    if (r->h_st->nan) {
      if (log) fprintf(log, "NaN in image! Exiting.\n");
      return IPG_E_NAN;
    }
    /* a pixel traced below is one the criterion flagged, never one it
     * interpolated, so the count taken before the trace stands */
    size_t total_interpolated = (size_t)r->h_st->interpolated;
    n = (size_t)r->h_st->n;
    if (n) {
      if ((rc = trace_level(ctx, cam, a, r, n, P, log))) return rc;
      traced += n;
    }
    size_t nxl = (size_t)a->params_nx / L.nsx, nyl = (size_t)a->params_ny / L.nsy;
    if (log)
      fprintf(log, "\n%zu of %zu (%f%%) of computed pixels at %zux%zu were interpolated\n\n", total_interpolated,
              nxl * nyl, ((double)total_interpolated) / (nxl * nyl) * 100, nxl, nyl);
  }

  CKR(cudaMemcpyAsync(img->image, r->image, npix * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(img->taus, r->taus, npix * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (!a->only_unpolarized)
    CKR(cudaMemcpyAsync(img->imageS, r->imageS, npix * NIMG * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(img->interp_flag, r->interp, npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(img->oddflag, r->oddflag, npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(img->nstep, r->nstep, npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CKR(cudaStreamSynchronize(s));
  img->traced = traced;
  return IPG_OK;
}

/* ================================================================ batches */
/* ipg_render_batch: the image driver above for many instances at once.  Per
 * level, every instance decides which of its candidate pixels to trace
 * exactly as a single image does (k_level with its own flux estimate and
 * keys); the instances of a camera group share the candidates, so the union
 * of their decisions is the group's list of geodesic items, each tagged with
 * the mask of the instance slots that trace it, and every instance's own
 * row-major list becomes its transfer items.  One ipg__batch_trace call
 * traces the level of all groups; save_pixel, the checks and the flux
 * estimate then run per instance on its share of the outputs. */

__global__ void k_fill_i32(int32_t *a, int n, int v)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) a[t] = v;
}

/* mask[t]: bit k set when instance slot k of the group traces candidate t */
__global__ void k_union(const int32_t *flags0, size_t stride, int G, int n, uint32_t *mask, int32_t *nz)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t m = 0;
  for (int k = 0; k < G; k++)
    if (flags0[(size_t)k * stride + t]) m |= 1u << k;
  mask[t] = m;
  nz[t] = m != 0;
}

/* the group's geodesic items in candidate order, and each candidate's
 * position among them */
__global__ void __launch_bounds__(SCAN_TPB) k_union_scatter(const uint32_t *mask, const int32_t *nz, int n,
                                                            const int32_t *block_sums, int nj, int nsx, int nsy,
                                                            int g, int32_t *geo_ij, int32_t *geo_grp,
                                                            uint32_t *geo_mask, int32_t *upos)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int f = t < n ? nz[t] : 0;
  int e = block_exclusive_scan(f, NULL);
  if (f) {
    int pos = block_sums[blockIdx.x] + e;
    geo_ij[2 * pos] = (t / nj) * nsx;
    geo_ij[2 * pos + 1] = (t % nj) * nsy;
    geo_grp[pos] = g;
    geo_mask[pos] = mask[t];
    upos[t] = pos;
  }
}

/* an instance's traced pixels -> their geodesic items */
__global__ void k_xf_map(const int32_t *ij, int n, int nj, int nsx, int nsy, const int32_t *upos, int geo_off,
                         int slot, int32_t *xf_geo, int32_t *xf_slot)
{
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  int t = (ij[2 * m] / nsx) * nj + ij[2 * m + 1] / nsy;
  xf_geo[m] = geo_off + upos[t];
  xf_slot[m] = slot;
}

/* The transfer order: items grouped by geodesic item, by slot within it, so
 * that the instances that trace one pixel sit in adjacent lanes and walk its
 * records in step (one load of the shared record serves them all, and their
 * coefficient blocks are contiguous); the geodesic items in the order their
 * geodesics start (longest predicted first).  cnt[r] = instances tracing the
 * r-th item of that order; off = its exclusive scan; order[off[rank of g] +
 * rank of the slot] = item. */
__global__ void k_geo_count(const uint32_t *mask, const int32_t *sorted, int n, int32_t *cnt, int32_t *rank)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) {
    const int g = sorted[t];
    cnt[t] = __popc(mask[g]);
    rank[g] = t;
  }
}

__global__ void __launch_bounds__(SCAN_TPB) k_geo_offsets(const int32_t *cnt, int n, const int32_t *block_sums,
                                                          int32_t *off)
{
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int e = block_exclusive_scan(t < n ? cnt[t] : 0, NULL);
  if (t < n) off[t] = block_sums[blockIdx.x] + e;
}

__global__ void k_xf_order(const int32_t *xf_geo, const int32_t *xf_slot, const uint32_t *mask, const int32_t *off,
                           const int32_t *rank, int n, int32_t *order)
{
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  const int g = xf_geo[m], k = xf_slot[m];
  order[off[rank[g]] + __popc(mask[g] & ((1u << k) - 1u))] = m;
}

namespace {
/* bump allocation inside one device block (a first pass only sizes it) */
struct Arena {
  char *base = nullptr;
  size_t off = 0;
  template <class T>
  T *take(size_t n)
  {
    size_t a = (off + 255) & ~(size_t)255;
    off = a + n * sizeof(T);
    return base ? reinterpret_cast<T *>(base + a) : nullptr;
  }
};

struct BInst {
  double *image, *taus, *imageS, *prelim;
  int32_t *interp, *oddflag, *nstep, *flags, *bsums, *winner;
  size_t npix, nprelim, traced;
  int grp, slot, set;
};

struct BGrp {
  int first, G; /* its instances are [first, first + G) in the internal order */
  uint32_t *mask;
  int32_t *nz, *bsums, *upos;
  int sx, sy, nx, ny, nxmin, nymin, levels;
};

bool same_camera(const ipg_instance &a, const ipg_instance &b)
{
  const ipg_camera &x = a.cam, &y = b.cam;
  return !memcmp(x.Xcam, y.Xcam, sizeof(x.Xcam)) && !memcmp(x.Econ, y.Econ, sizeof(x.Econ)) &&
         !memcmp(x.Ecov, y.Ecov, sizeof(x.Ecov)) && x.fovx == y.fovx && x.fovy == y.fovy && x.rotcam == y.rotcam &&
         x.xoff == y.xoff && x.yoff == y.yoff && x.freq == y.freq && x.eps == y.eps && x.nx == y.nx &&
         x.ny == y.ny && x.maxnstep == y.maxnstep && x.only_unpolarized == y.only_unpolarized &&
         x.emission_type == y.emission_type && x.stokes_floors == y.stokes_floors &&
         x.target_nturns == y.target_nturns && x.subring_dtheta == y.subring_dtheta && x.counterjet == y.counterjet &&
         a.nx == b.nx && a.ny == b.ny && a.nx_min == b.nx_min && a.ny_min == b.ny_min &&
         a.refine_level == b.refine_level;
}

bool same_electrons(const ipg_electrons &a, const ipg_electrons &b)
{
  return a.RHO_unit == b.RHO_unit && a.B_unit == b.B_unit && a.trat_large == b.trat_large &&
         a.trat_small == b.trat_small && a.beta_crit == b.beta_crit;
}
} // namespace

struct BatchArena {
  void *dev = nullptr;
  size_t bytes = 0;
};

extern "C" void ipg__batch_arena_release(void *p)
{
  BatchArena *a = (BatchArena *)p;
  if (!a) return;
  cudaFree(a->dev);
  delete a;
}

extern "C" int ipg_render_batch(ipg_ctx *ctx, const ipg_instance *inst, size_t n, ipg_instance_image *outs,
                                uint64_t step_budget)
{
  if (!ctx || !inst || !outs || n == 0) return IPG_E_ARG;
  if (n > (size_t)IPG_BATCH_MAX_CAMERAS * IPG_BATCH_MAX_PER_CAMERA) return IPG_E_ARG;
  cudaStream_t s = (cudaStream_t)ipg__stream(ctx);
  /* camera groups and electron models */
  std::vector<int> grp_of(n), set_of(n);
  std::vector<int> grp_rep, set_rep;
  int maxnstep_all = 2; /* the step cap of the length prediction */
  for (size_t i = 0; i < n; i++) {
    const ipg_instance &a = inst[i];
    if (a.cam.maxnstep > maxnstep_all) maxnstep_all = a.cam.maxnstep;
    if (a.nx < 2 || a.ny < 2 || a.nx_min < 2 || a.ny_min < 2 || a.refine_level < 1 || !outs[i].image ||
        !outs[i].taus || !outs[i].interp_flag || !outs[i].oddflag || !outs[i].nstep ||
        (!a.cam.only_unpolarized && !outs[i].imageS) || (size_t)a.nx * a.ny >= (size_t)INT_MAX / 2)
      return IPG_E_ARG;
    int g = -1;
    for (size_t q = 0; q < grp_rep.size(); q++)
      if (same_camera(inst[grp_rep[q]], a)) g = (int)q;
    if (g < 0) {
      g = (int)grp_rep.size();
      grp_rep.push_back((int)i);
    }
    grp_of[i] = g;
    int e = -1;
    for (size_t q = 0; q < set_rep.size(); q++)
      if (same_electrons(inst[set_rep[q]].el, a.el)) e = (int)q;
    if (e < 0) {
      e = (int)set_rep.size();
      set_rep.push_back((int)i);
    }
    set_of[i] = e;
  }
  const int ngrp = (int)grp_rep.size();
  if (ngrp > IPG_BATCH_MAX_CAMERAS) {
    ipg__set_error(ctx, "too many camera groups in one batch");
    return IPG_E_ARG;
  }
  /* internal order: instances grouped by camera, slots in input order */
  std::vector<int> order;
  std::vector<BGrp> grps(ngrp);
  int G = 1;
  for (int g = 0; g < ngrp; g++) {
    grps[g].first = (int)order.size();
    for (size_t i = 0; i < n; i++)
      if (grp_of[i] == g) order.push_back((int)i);
    grps[g].G = (int)order.size() - grps[g].first;
    if (grps[g].G > IPG_BATCH_MAX_PER_CAMERA) {
      ipg__set_error(ctx, "more than IPG_BATCH_MAX_PER_CAMERA instances share one camera");
      return IPG_E_ARG;
    }
    if (grps[g].G > G) G = grps[g].G;
    const ipg_instance &r = inst[grp_rep[g]];
    grps[g].nx = r.nx;
    grps[g].ny = r.ny;
    grps[g].nxmin = r.nx_min;
    grps[g].nymin = r.ny_min;
    grps[g].sx = (r.nx - 1) / (r.nx_min - 1);
    grps[g].sy = (r.ny - 1) / (r.ny_min - 1);
    grps[g].levels = r.refine_level;
  }
  std::vector<ipg_camera> gcam(ngrp);
  std::vector<int> slot_set((size_t)ngrp * G, 0);
  for (int g = 0; g < ngrp; g++) {
    gcam[g] = inst[grp_rep[g]].cam;
    for (int k = 0; k < grps[g].G; k++) slot_set[(size_t)g * G + k] = set_of[order[grps[g].first + k]];
  }
  std::vector<ipg_electrons> sets(set_rep.size());
  for (size_t e = 0; e < set_rep.size(); e++) sets[e] = inst[set_rep[e]].el;
  int rc = ipg__batch_begin(ctx, gcam.data(), ngrp, slot_set.data(), G, sets.data(), (int)sets.size(),
                            ipg__step32(ctx));
  if (rc) return rc;

  /* device memory: per instance its image and level buffers, per group its
   * union buffers, and the items of the largest level */
  std::vector<BInst> bi(n);
  size_t sum_pix = 0, sum_gpix = 0;
  for (size_t q = 0; q < n; q++) {
    const ipg_instance &a = inst[order[q]];
    bi[q].npix = (size_t)a.nx * a.ny;
    bi[q].nprelim = a.refine_level > 1 ? (size_t)a.nx_min * a.ny_min : 1;
    bi[q].grp = grp_of[order[q]];
    bi[q].slot = (int)q - grps[bi[q].grp].first;
    bi[q].set = set_of[order[q]];
    bi[q].traced = 0;
    sum_pix += bi[q].npix;
  }
  for (int g = 0; g < ngrp; g++) sum_gpix += (size_t)grps[g].nx * grps[g].ny;
  BatchArena **slot = (BatchArena **)ipg__batch_arena_slot(ctx);
  if (!*slot) *slot = new BatchArena();
  BatchArena *ar = *slot;
  Arena A;
  RefineStatus *st = nullptr, *gst = nullptr;
  int32_t *ij_all = nullptr, *xf_geo = nullptr, *xf_slot = nullptr, *geo_ij = nullptr, *geo_grp = nullptr;
  uint32_t *geo_mask = nullptr;
  int32_t *geo_cnt = nullptr, *geo_bsums = nullptr, *geo_off = nullptr, *xf_order = nullptr;
  int32_t *geo_sorted = nullptr, *geo_rank = nullptr, *geo_pred = nullptr;
  RefineStatus *ord_st = nullptr;
  ipg_pixel_out *xf_out = nullptr;
  std::vector<int32_t *> gflags(ngrp);
  for (int pass = 0; pass < 2; pass++) {
    A.base = pass ? (char *)ar->dev : nullptr;
    A.off = 0;
    for (size_t q = 0; q < n; q++) {
      BInst &b = bi[q];
      b.image = A.take<double>(b.npix);
      b.taus = A.take<double>(b.npix);
      b.imageS = gcam[b.grp].only_unpolarized ? nullptr : A.take<double>(b.npix * NIMG);
      b.interp = A.take<int32_t>(b.npix);
      b.oddflag = A.take<int32_t>(b.npix);
      b.nstep = A.take<int32_t>(b.npix);
      b.bsums = A.take<int32_t>(b.npix / SCAN_TPB + 2);
      b.prelim = A.take<double>(b.nprelim);
      b.winner = A.take<int32_t>(b.nprelim);
    }
    for (int g = 0; g < ngrp; g++) {
      size_t gp = (size_t)grps[g].nx * grps[g].ny;
      /* the candidate flags of the group's instances, one row each */
      gflags[g] = A.take<int32_t>(gp * grps[g].G);
      for (int k = 0; k < grps[g].G; k++) bi[grps[g].first + k].flags = gflags[g] ? gflags[g] + gp * k : nullptr;
      grps[g].mask = A.take<uint32_t>(gp);
      grps[g].nz = A.take<int32_t>(gp);
      grps[g].bsums = A.take<int32_t>(gp / SCAN_TPB + 2);
      grps[g].upos = A.take<int32_t>(gp);
    }
    st = A.take<RefineStatus>(n);
    gst = A.take<RefineStatus>(ngrp);
    ij_all = A.take<int32_t>(2 * sum_pix);
    xf_geo = A.take<int32_t>(sum_pix);
    xf_slot = A.take<int32_t>(sum_pix);
    xf_out = A.take<ipg_pixel_out>(sum_pix);
    geo_ij = A.take<int32_t>(2 * sum_gpix);
    geo_grp = A.take<int32_t>(sum_gpix);
    geo_mask = A.take<uint32_t>(sum_gpix);
    geo_cnt = A.take<int32_t>(sum_gpix);
    geo_bsums = A.take<int32_t>(sum_gpix / SCAN_TPB + 2);
    geo_off = A.take<int32_t>(sum_gpix);
    xf_order = A.take<int32_t>(sum_pix);
    ord_st = A.take<RefineStatus>(1);
    geo_sorted = A.take<int32_t>(sum_gpix);
    geo_rank = A.take<int32_t>(sum_gpix);
    geo_pred = A.take<int32_t>(sum_gpix);
    if (pass == 0 && ar->bytes < A.off) {
      cudaFree(ar->dev);
      ar->dev = nullptr;
      ar->bytes = 0;
      CKR(cudaMalloc(&ar->dev, A.off));
      ar->bytes = A.off;
    }
  }
  for (size_t q = 0; q < n; q++) {
    BInst &b = bi[q];
    CKR(cudaMemsetAsync(b.image, 0, b.npix * sizeof(double), s));
    CKR(cudaMemsetAsync(b.taus, 0, b.npix * sizeof(double), s));
    if (b.imageS) CKR(cudaMemsetAsync(b.imageS, 0, b.npix * NIMG * sizeof(double), s));
    CKR(cudaMemsetAsync(b.interp, 0, b.npix * sizeof(int32_t), s));
    CKR(cudaMemsetAsync(b.oddflag, 0, b.npix * sizeof(int32_t), s));
    CKR(cudaMemsetAsync(b.nstep, 0, b.npix * sizeof(int32_t), s));
  }
  {
    std::vector<RefineStatus> z(n);
    for (auto &x : z) {
      memset(&x, 0, sizeof(x));
      x.maxn_first = INT_MAX;
    }
    CKR(cudaMemcpyAsync(st, z.data(), n * sizeof(RefineStatus), cudaMemcpyHostToDevice, s));
  }
  unsigned long long steps_left = step_budget;
  std::vector<RefineStatus> hst(n), hgst(ngrp);
  std::vector<size_t> nlist(n), xoff(n), goff(ngrp), ucount(ngrp);
  int maxlev = 0;
  for (int g = 0; g < ngrp; g++) maxlev = grps[g].levels > maxlev ? grps[g].levels : maxlev;

  for (int lvl = 0; lvl < maxlev; lvl++) {
    std::vector<LevelArgs> L(ngrp);
    std::vector<int> active(ngrp, 0);
    for (int g = 0; g < ngrp; g++) {
      BGrp &gr = grps[g];
      if (lvl >= gr.levels) continue;
      active[g] = 1;
      LevelArgs &l = L[g];
      memset(&l, 0, sizeof(l));
      l.nx = gr.nx;
      l.ny = gr.ny;
      if (lvl == 0) {
        l.nsx = gr.sx;
        l.nsy = gr.sy;
      } else {
        l.nsx = (int)(gr.sx / pow(2, lvl));
        l.nsy = (int)(gr.sy / pow(2, lvl));
        if (l.nsx < 1 || l.nsy < 1) {
          ipg__set_error(ctx, "refinement spacing below one pixel: nx_min/ny_min too small");
          return IPG_E_ARG;
        }
      }
      l.psx = 2 * l.nsx;
      l.psy = 2 * l.nsy;
      l.ni = (gr.nx - 1) / l.nsx + 1;
      l.nj = (gr.ny - 1) / l.nsy + 1;
    }
    /* every instance's decisions and its own list count */
    for (size_t q = 0; q < n; q++) {
      BInst &b = bi[q];
      if (!active[b.grp]) continue;
      const ipg_instance &a = inst[order[q]];
      LevelArgs l = L[b.grp];
      l.unpol = a.cam.only_unpolarized;
      l.nearest = a.nearest_neighbor;
      l.refine_abs = a.refine_abs;
      l.refine_rel = a.refine_rel;
      l.refine_cut = a.refine_cut;
      const int ncand = l.ni * l.nj, nb = grid_of(ncand, SCAN_TPB);
      RefineStatus zz;
      memset(&zz, 0, sizeof(zz));
      zz.maxn_first = INT_MAX;
      /* keep Iavg: the levels read it */
      CKR(cudaMemcpyAsync(st + q, &zz, offsetof(RefineStatus, Iavg), cudaMemcpyHostToDevice, s));
      ImgPtrs P = {b.image, b.taus, b.imageS, b.interp, b.oddflag, b.nstep, a.ny};
      if (lvl == 0) k_fill_i32<<<grid_of(ncand, TPB), TPB, 0, s>>>(b.flags, ncand, 1);
      else k_level<<<grid_of(ncand, TPB), TPB, 0, s>>>(l, P, st + q, b.flags, st + q);
      k_scan_blocks<<<nb, SCAN_TPB, 0, s>>>(b.flags, ncand, b.bsums);
      k_scan_top<<<1, SCAN_TPB, 0, s>>>(b.bsums, nb, st + q);
    }
    /* the groups' unions */
    for (int g = 0; g < ngrp; g++) {
      if (!active[g]) continue;
      BGrp &gr = grps[g];
      const int ncand = L[g].ni * L[g].nj, nb = grid_of(ncand, SCAN_TPB);
      const size_t stride = (size_t)gr.nx * gr.ny;
      k_union<<<grid_of(ncand, TPB), TPB, 0, s>>>(gflags[g], stride, gr.G, ncand, gr.mask, gr.nz);
      k_scan_blocks<<<nb, SCAN_TPB, 0, s>>>(gr.nz, ncand, gr.bsums);
      k_scan_top<<<1, SCAN_TPB, 0, s>>>(gr.bsums, nb, gst + g);
    }
    CKR(cudaGetLastError());
    CKR(cudaMemcpyAsync(hst.data(), st, n * sizeof(RefineStatus), cudaMemcpyDeviceToHost, s));
    CKR(cudaMemcpyAsync(hgst.data(), gst, ngrp * sizeof(RefineStatus), cudaMemcpyDeviceToHost, s));
    CKR(cudaStreamSynchronize(s));
    size_t n_geo = 0, n_xf = 0;
    for (int g = 0; g < ngrp; g++) {
      goff[g] = n_geo;
      ucount[g] = active[g] ? (size_t)hgst[g].n : 0;
      n_geo += ucount[g];
    }
    for (size_t q = 0; q < n; q++) {
      nlist[q] = 0;
      if (!active[bi[q].grp]) continue;
      if (hst[q].nan) {
        char m[128];
        snprintf(m, sizeof(m), "NaN in the image of batch instance %d", order[q]);
        ipg__set_error(ctx, m);
        return IPG_E_NAN;
      }
      xoff[q] = n_xf;
      nlist[q] = (size_t)hst[q].n;
      n_xf += nlist[q];
    }
    if (n_geo == 0) continue;
    for (int g = 0; g < ngrp; g++) {
      if (!active[g] || !ucount[g]) continue;
      const int ncand = L[g].ni * L[g].nj, nb = grid_of(ncand, SCAN_TPB);
      k_union_scatter<<<nb, SCAN_TPB, 0, s>>>(grps[g].mask, grps[g].nz, ncand, grps[g].bsums, L[g].nj, L[g].nsx,
                                               L[g].nsy, g, geo_ij + 2 * goff[g], geo_grp + goff[g],
                                               geo_mask + goff[g], grps[g].upos);
    }
    for (size_t q = 0; q < n; q++) {
      if (!nlist[q]) continue;
      const BInst &b = bi[q];
      const LevelArgs &l = L[b.grp];
      const int ncand = l.ni * l.nj, nb = grid_of(ncand, SCAN_TPB);
      k_scatter<<<nb, SCAN_TPB, 0, s>>>(b.flags, ncand, b.bsums, l.nj, l.nsx, l.nsy, ij_all + 2 * xoff[q]);
      k_xf_map<<<grid_of((long long)nlist[q], TPB), TPB, 0, s>>>(ij_all + 2 * xoff[q], (int)nlist[q], l.nj, l.nsx,
                                                                  l.nsy, grps[b.grp].upos, (int)goff[b.grp], b.slot,
                                                                  xf_geo + xoff[q], xf_slot + xoff[q]);
    }
    size_t n_long = 0;
    double long_steps = 0., pred_steps = 0.;
    {
      const int ng = (int)n_geo, nb = grid_of(ng, SCAN_TPB);
      if ((rc = ipg__batch_sort_geo(ctx, geo_ij, geo_grp, n_geo, maxnstep_all, geo_pred, geo_sorted, &n_long,
                                    &long_steps, &pred_steps)))
        return rc;
      k_geo_count<<<grid_of(ng, TPB), TPB, 0, s>>>(geo_mask, geo_sorted, ng, geo_cnt, geo_rank);
      k_scan_blocks<<<nb, SCAN_TPB, 0, s>>>(geo_cnt, ng, geo_bsums);
      k_scan_top<<<1, SCAN_TPB, 0, s>>>(geo_bsums, nb, ord_st);
      k_geo_offsets<<<nb, SCAN_TPB, 0, s>>>(geo_cnt, ng, geo_bsums, geo_off);
      if (n_xf) k_xf_order<<<grid_of((long long)n_xf, TPB), TPB, 0, s>>>(xf_geo, xf_slot, geo_mask, geo_off, geo_rank,
                                                                      (int)n_xf, xf_order);
    }
    CKR(cudaGetLastError());
    ipg_batch_items items = {n_geo,   geo_ij, geo_grp,  geo_mask,   n_xf,   xf_geo,
                             xf_slot, xf_out, xf_order, geo_sorted, n_long, long_steps, pred_steps};
    rc = ipg__batch_trace(ctx, &items, step_budget ? &steps_left : nullptr);
    if (rc) return rc;
    /* save_pixel, the checks and (base level) the flux estimate per instance */
    for (size_t q = 0; q < n; q++) {
      if (!nlist[q]) continue;
      BInst &b = bi[q];
      const ipg_instance &a = inst[order[q]];
      const int nq = (int)nlist[q];
      ImgPtrs P = {b.image, b.taus, b.imageS, b.interp, b.oddflag, b.nstep, a.ny};
      k_check<<<grid_of(nq, TPB), TPB, 0, s>>>(xf_out + xoff[q], nq, a.cam.maxnstep, a.cam.only_unpolarized, st + q);
      k_save<<<grid_of(nq, TPB), TPB, 0, s>>>(ij_all + 2 * xoff[q], xf_out + xoff[q], nq, P, a.f3,
                                              a.cam.only_unpolarized, a.qu_conv, st + q);
      if (lvl == 0 && a.refine_level > 1) {
        const long long nslot = (long long)b.nprelim;
        CKR(cudaMemsetAsync(b.prelim, 0, b.nprelim * sizeof(double), s));
        CKR(cudaMemsetAsync(b.winner, 0xff, b.nprelim * sizeof(int32_t), s));
        const BGrp &gr = grps[b.grp];
        k_prelim_claim<<<grid_of(nq, TPB), TPB, 0, s>>>(ij_all + 2 * xoff[q], nq, a.nx, a.ny, a.ny_min, gr.sx,
                                                        gr.sy, nslot, b.winner);
        k_prelim_fill<<<grid_of(nq, TPB), TPB, 0, s>>>(ij_all + 2 * xoff[q], xf_out + xoff[q], nq, a.nx, a.ny,
                                                       a.ny_min, gr.sx, gr.sy, nslot, b.winner, b.prelim);
        k_prelim_sum<<<1, 32, 0, s>>>(b.prelim, nslot, a.f3, (double)b.npix, st + q);
      }
      b.traced += nlist[q];
    }
    CKR(cudaGetLastError());
    CKR(cudaMemcpyAsync(hst.data(), st, n * sizeof(RefineStatus), cudaMemcpyDeviceToHost, s));
    CKR(cudaStreamSynchronize(s));
    for (size_t q = 0; q < n; q++) {
      if (!nlist[q]) continue;
      if (hst[q].maxn_first != INT_MAX) {
        int32_t pij[2];
        CKR(cudaMemcpy(pij, ij_all + 2 * (xoff[q] + (size_t)hst[q].maxn_first), sizeof(pij), cudaMemcpyDeviceToHost));
        char m[160];
        snprintf(m, sizeof(m), "MaxNStep exceeded in pixel %d %d of batch instance %d", pij[0], pij[1], order[q]);
        ipg__set_error(ctx, m);
        return IPG_E_MAXNSTEP;
      }
      if (hst[q].nan) {
        char m[128];
        snprintf(m, sizeof(m), "NaN in the image of batch instance %d", order[q]);
        ipg__set_error(ctx, m);
        return IPG_E_NAN;
      }
    }
  }
  for (size_t q = 0; q < n; q++) {
    const BInst &b = bi[q];
    ipg_instance_image &o = outs[order[q]];
    CKR(cudaMemcpyAsync(o.image, b.image, b.npix * sizeof(double), cudaMemcpyDeviceToHost, s));
    CKR(cudaMemcpyAsync(o.taus, b.taus, b.npix * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (b.imageS) CKR(cudaMemcpyAsync(o.imageS, b.imageS, b.npix * NIMG * sizeof(double), cudaMemcpyDeviceToHost, s));
    CKR(cudaMemcpyAsync(o.interp_flag, b.interp, b.npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CKR(cudaMemcpyAsync(o.oddflag, b.oddflag, b.npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CKR(cudaMemcpyAsync(o.nstep, b.nstep, b.npix * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    o.traced = b.traced;
  }
  CKR(cudaStreamSynchronize(s));
  return IPG_OK;
}
