// grid.cu -- substrate grid build on the device.
//
// Output: B-spline coefficients of (Pauli, London, Coulomb, 0) packed as float4 in the
// z-fastest layout i = iz + nz*(iy + ny*ix) that the relaxation kernel samples.
//
//   Morse channels .... Pauli = sum_j E_j exp(-2a(r - R_j)), London = sum_j -2 E_j exp(-a(r - R_j))
//                       over ions and (2 npbc + 1)^2 lateral images (opencl/gridff_build.cl:217-347,
//                       make_MorseFF); FP32 terms, FP64 accumulation.
//   Coulomb channel ... Ewald-2D for a slab below the grid (opencl/Surface.cl:716-906):
//                         phi = K [ -(2pi/A) sum_i q_i (z - z_i)
//                                   + Re sum_{G != 0} (2pi/(A|G|)) S_G exp(iG.rho) exp(-|G|(z - z0)) ]
//                       with S_G = sum_i q_i exp(-iG.rho_i) exp(-|G|(z0 - z_i)), all in FP64.  S_G is
//                       built per ion layer from separable phase tables; phi on each z plane is a
//                       two-stage partial DFT (over h, then over k), skipping G whose amplitude is
//                       below ewald_tol of the largest.
//   B-spline fit ...... exact solution of Conv(c) = V for the forward operator of BsplineConv3D
//                       (opencl/gridff_build.cl:8-61): separable tridiag(1/6, 2/3, 1/6) solves, cyclic
//                       (Sherman-Morrison) in x and y, zero-padded in z; FP64.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "smr_internal.h"
#include "../../include/surfmol_relax.h"

namespace smr {
namespace {

constexpr double kCoulombD = 14.3996448915;
constexpr double kPi = 3.14159265358979323846;

#define GB_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { std::snprintf(err, errlen, "%s: %s", #x, cudaGetErrorString(e_)); return -1; } } while (0)

// ---------------------------------------------------------------- Morse
// x-planes [x0, x0 + xs) of the grid; outputs indexed within that slab (z-fastest)
__global__ void morse_kernel(int nions, const double* __restrict__ ions, const double* __restrict__ re,
                             double Lx, double Ly, int npbc, int x0, int xs, int ny, int nz, double p0x, double p0y, double p0z,
                             double sx, double sy, double sz, float alpha, float rcut2, double* __restrict__ paul,
                             double* __restrict__ lond) {
    __shared__ float4 sI[128];
    __shared__ float2 sR[128];
    const size_t N = (size_t)xs * ny * nz;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = idx < N;
    const int iz = (int)(idx % nz), iy = (int)((idx / nz) % ny), ix = x0 + (int)(idx / ((size_t)nz * ny));
    // grid point relative coordinates in FP64, then FP32 per term
    const double px = p0x + ix * sx, py = p0y + iy * sy, pz = p0z + iz * sz;
    double P = 0.0, Lo = 0.0;
    for (int j0 = 0; j0 < nions; j0 += 128) {
        const int j = j0 + threadIdx.x;
        if (threadIdx.x < 128) {
            if (j < nions) {
                sI[threadIdx.x] = make_float4((float)ions[4 * j], (float)ions[4 * j + 1], (float)ions[4 * j + 2], 0.f);
                sR[threadIdx.x] = make_float2((float)re[4 * j], (float)re[4 * j + 1]);
            }
        }
        __syncthreads();
        const int m = min(128, nions - j0);
        if (live) {
            for (int k = 0; k < m; k++) {
                const float4 a = sI[k];
                const float2 r = sR[k];
                // displacement to the nearest copy handled by summing all images explicitly
                const float dx0 = (float)(px - (double)a.x), dy0 = (float)(py - (double)a.y), dz = (float)(pz - (double)a.z);
                float sp = 0.f, sl = 0.f;
                for (int jy = -npbc; jy <= npbc; jy++)
                    for (int jx = -npbc; jx <= npbc; jx++) {
                        const float dx = dx0 + jx * (float)Lx, dy = dy0 + jy * (float)Ly;
                        const float r2 = dx * dx + dy * dy + dz * dz;
                        if (r2 > rcut2) continue;
                        const float rr = sqrtf(r2 + 1e-32f);
                        const float e = expf(-alpha * (rr - r.x));
                        const float eM = r.y * e;
                        sp += eM * e;
                        sl += -2.0f * eM;
                    }
                P += (double)sp; Lo += (double)sl;
            }
        }
        __syncthreads();
    }
    if (live) { paul[idx] = P; lond[idx] = Lo; }
}

// ---------------------------------------------------------------- Ewald-2D
// phase tables: X[i*(2H+1) + (h+H)] = exp(-i h g1 x_i), Y[i*(2K+1) + (k+K)] = exp(-i k g2 y_i)
__global__ void phase_table_kernel(int nions, const double* __restrict__ ions, int comp, double g, int H, double2* __restrict__ X) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int w = 2 * H + 1;
    if (t >= nions * w) return;
    const int i = t / w, h = t % w - H;
    double s, c;
    sincos(-(double)h * g * ions[4 * i + comp], &s, &c);
    X[t] = make_double2(c, s);
}

// S[(k+K)*(2H+1) + (h+H)] = sum_layers exp(-|G| d_l) sum_{i in l} q_i X_i(h) Y_i(k)
__global__ void structure_factor_kernel(int nions, const double* __restrict__ ions, const double* __restrict__ dz_ion,
                                        const double2* __restrict__ X, const double2* __restrict__ Y, int H, int K,
                                        double g1, double g2, double2* __restrict__ S) {
    const int w = 2 * H + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= w * (2 * K + 1)) return;
    const int hh = t % w, kk = t / w;
    const double Gx = (hh - H) * g1, Gy = (kk - K) * g2, Gn = sqrt(Gx * Gx + Gy * Gy);
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < nions; i++) {
        const double2 a = X[(size_t)i * w + hh];
        const double2 b = Y[(size_t)i * (2 * K + 1) + kk];
        const double q = ions[4 * i + 3] * exp(-Gn * dz_ion[i]);
        sr += q * (a.x * b.x - a.y * b.y);
        si += q * (a.x * b.y + a.y * b.x);
    }
    S[t] = make_double2(sr, si);
}

// phase table out[r*n + i] = exp(i m_r g (p0 + i s)) for integer multipliers m_r
__global__ void line_phase_kernel(int nrows, const int* __restrict__ mult, int n, double p0, double st, double g,
                                  double2* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows * n) return;
    const int r = t / n, i = t % n;
    double s, c;
    sincos((double)mult[r] * g * (p0 + i * st), &s, &c);
    out[t] = make_double2(c, s);
}

// amplitudes of one z plane: amp0 * exp(-|G| (z - z0)), zeroed below the pruning threshold
__global__ void plane_amp_kernel(int ne, const double2* __restrict__ amp0, const double* __restrict__ gnorm, double dzp,
                                 double thresh, double2* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const double d = exp(-gnorm[e] * dzp);
    const double2 a = amp0[e];
    out[e] = ((fabs(a.x) + fabs(a.y)) * d < thresh) ? make_double2(0.0, 0.0) : make_double2(a.x * d, a.y * d);
}

// Stage 1: B[r*nx + ix] = sum_{e in row r} amp[e] * Ex[hidx[e]*nx + ix]
__global__ void ewald_stage1(int nrows, const int* __restrict__ rowptr, const int* __restrict__ hidx,
                             const double2* __restrict__ amp, const double2* __restrict__ Ex, int nx, double2* __restrict__ B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nrows * nx) return;
    const int r = t / nx, ix = t % nx;
    double br = 0.0, bi = 0.0;
    for (int e = rowptr[r]; e < rowptr[r + 1]; e++) {
        const double2 a = amp[e];
        const double2 c = Ex[(size_t)hidx[e] * nx + ix];
        br += a.x * c.x - a.y * c.y;
        bi += a.x * c.y + a.y * c.x;
    }
    B[t] = make_double2(br, bi);
}

// Stage 2: phi(ix, iy) = K (phi0 + Re sum_r B[r, ix] Ey[r, iy])
// x-planes [x0, x0 + xs) of plane iz; B holds the x factors of all nx planes
__global__ void ewald_stage2(int nrows, const double2* __restrict__ B, const double2* __restrict__ Ey, int nx, int ny,
                             int x0, int xs, double phi0, int iz, int nz, double* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= xs * ny) return;
    const int iy = t % ny, lx = t / ny, ix = x0 + lx;
    double acc = 0.0;
    for (int r = 0; r < nrows; r++) {
        const double2 b = B[(size_t)r * nx + ix];
        const double2 c = Ey[(size_t)r * ny + iy];
        acc += b.x * c.x - b.y * c.y;
    }
    out[(size_t)iz + (size_t)nz * ((size_t)iy + (size_t)ny * lx)] = kCoulombD * (phi0 + acc);
}

// ---------------------------------------------------------------- B-spline fit
// Line solve of tridiag(a, b, a) x = d with precomputed forward coefficients cp[] and
// pivots m[]: d'[0] = d[0]/m[0], d'[i] = (d[i] - a d'[i-1]) / m[i]; x[i] = d'[i] - cp[i] x[i+1].
__device__ __forceinline__ void thomas_line(double* x, size_t st, int n, const double* cp, const double* m) {
    const double a = 1.0 / 6.0;
    double prev = x[0] / m[0];
    x[0] = prev;
    for (int i = 1; i < n; i++) { prev = (x[(size_t)i * st] - a * prev) / m[i]; x[(size_t)i * st] = prev; }
    double nxt = x[(size_t)(n - 1) * st];
    for (int i = n - 2; i >= 0; i--) { nxt = x[(size_t)i * st] - cp[i] * nxt; x[(size_t)i * st] = nxt; }
}

// periodic correction: x -= fact * u with fact = (x0 + a x_{n-1}/gamma) / den
__device__ __forceinline__ void cyclic_fix(double* x, size_t st, int n, const double* u, double gamma, double den) {
    const double a = 1.0 / 6.0;
    const double fact = (x[0] + a * x[(size_t)(n - 1) * st] / gamma) / den;
    for (int i = 0; i < n; i++) x[(size_t)i * st] -= fact * u[i];
}

struct LineCoef { double* cp; double* m; double* u; double gamma, den; int n; bool periodic; };

__global__ void fit_z(double* v, int nx, int ny, int nz, const double* cp, const double* m) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nx * ny) return;
    thomas_line(v + (size_t)t * nz, 1, nz, cp, m);
}
__global__ void fit_y(double* v, int nx, int ny, int nz, const double* cp, const double* m, const double* u, double gamma, double den) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nx * nz) return;
    const int iz = t % nz, ix = t / nz;
    double* x = v + iz + (size_t)nz * ny * ix;
    thomas_line(x, nz, ny, cp, m);
    cyclic_fix(x, nz, ny, u, gamma, den);
}
__global__ void fit_x(double* v, int nx, int ny, int nz, const double* cp, const double* m, const double* u, double gamma, double den) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ny * nz) return;
    const int iz = t % nz, iy = t / nz;
    double* x = v + iz + (size_t)nz * iy;
    thomas_line(x, (size_t)nz * ny, nx, cp, m);
    cyclic_fix(x, (size_t)nz * ny, nx, u, gamma, den);
}

__global__ void pack_kernel(size_t N, const double* __restrict__ c0, const double* __restrict__ c1, const double* __restrict__ c2,
                            float4* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    out[i] = make_float4((float)c0[i], (float)c1[i], (float)c2[i], 0.f);
}

// host: Thomas coefficients of tridiag(1/6, b0|2/3..|bn, 1/6)
void thomas_coefs(int n, double b0, double bn, std::vector<double>& cp, std::vector<double>& m) {
    const double a = 1.0 / 6.0, b = 2.0 / 3.0;
    cp.assign(n, 0.0); m.assign(n, 0.0);
    m[0] = b0; cp[0] = a / m[0];
    for (int i = 1; i < n; i++) {
        const double di = (i == n - 1) ? bn : b;
        m[i] = di - a * cp[i - 1];
        cp[i] = a / m[i];
    }
}
void thomas_host(std::vector<double>& x, const std::vector<double>& cp, const std::vector<double>& m) {
    const double a = 1.0 / 6.0;
    int n = (int)x.size();
    x[0] /= m[0];
    for (int i = 1; i < n; i++) x[i] = (x[i] - a * x[i - 1]) / m[i];
    for (int i = n - 2; i >= 0; i--) x[i] -= cp[i] * x[i + 1];
}

struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() { for (void* p : ptrs) cudaFree(p); }
    template <class T> cudaError_t alloc(T** p, size_t n) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

int fit_channel(double* d, int nx, int ny, int nz, cudaStream_t s, DevBuf& buf, char* err, int errlen) {
    const double a = 1.0 / 6.0, b = 2.0 / 3.0;
    // z: open (zero padded)
    {
        std::vector<double> cp, m;
        thomas_coefs(nz, b, b, cp, m);
        double *dcp, *dm;
        GB_CHECK(buf.alloc(&dcp, nz)); GB_CHECK(buf.alloc(&dm, nz));
        GB_CHECK(cudaMemcpyAsync(dcp, cp.data(), nz * 8, cudaMemcpyHostToDevice, s));
        GB_CHECK(cudaMemcpyAsync(dm, m.data(), nz * 8, cudaMemcpyHostToDevice, s));
        fit_z<<<(nx * ny + 127) / 128, 128, 0, s>>>(d, nx, ny, nz, dcp, dm);
        GB_CHECK(cudaGetLastError());
        GB_CHECK(cudaStreamSynchronize(s));
    }
    // y and x: cyclic, gamma = -b (tridiagonal part with modified corners + rank-one correction)
    for (int axis = 0; axis < 2; axis++) {
        const int n = axis == 0 ? ny : nx;
        const double gamma = -b;
        std::vector<double> cp, m, u(n, 0.0);
        thomas_coefs(n, b - gamma, b - a * a / gamma, cp, m);
        u[0] = gamma; u[n - 1] = a;
        thomas_host(u, cp, m);
        const double den = 1.0 + u[0] + a * u[n - 1] / gamma;
        double *dcp, *dm, *du;
        GB_CHECK(buf.alloc(&dcp, n)); GB_CHECK(buf.alloc(&dm, n)); GB_CHECK(buf.alloc(&du, n));
        GB_CHECK(cudaMemcpyAsync(dcp, cp.data(), n * 8, cudaMemcpyHostToDevice, s));
        GB_CHECK(cudaMemcpyAsync(dm, m.data(), n * 8, cudaMemcpyHostToDevice, s));
        GB_CHECK(cudaMemcpyAsync(du, u.data(), n * 8, cudaMemcpyHostToDevice, s));
        if (axis == 0) fit_y<<<(nx * nz + 127) / 128, 128, 0, s>>>(d, nx, ny, nz, dcp, dm, du, gamma, den);
        else fit_x<<<(ny * nz + 127) / 128, 128, 0, s>>>(d, nx, ny, nz, dcp, dm, du, gamma, den);
        GB_CHECK(cudaGetLastError());
        GB_CHECK(cudaStreamSynchronize(s));
    }
    return 0;
}

// ---------------------------------------------------------------- 16-bit encoding
// per (z plane, channel) max |c|: each block reduces a contiguous voxel range into shared memory
// (voxel i lies on plane i % nz), then merges into the global table
__global__ void plane_absmax_kernel(size_t N, int nz, const float4* __restrict__ src, unsigned int* __restrict__ mx) {
    extern __shared__ unsigned int sm[];
    for (int k = threadIdx.x; k < 4 * nz; k += blockDim.x) sm[k] = 0u;
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = src[i];
        const int z = (int)(i % (size_t)nz);
        atomicMax(sm + 4 * z + 0, __float_as_uint(fabsf(v.x)));    // non-negative floats order as uints
        atomicMax(sm + 4 * z + 1, __float_as_uint(fabsf(v.y)));
        atomicMax(sm + 4 * z + 2, __float_as_uint(fabsf(v.z)));
        atomicMax(sm + 4 * z + 3, __float_as_uint(fabsf(v.w)));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 4 * nz; k += blockDim.x)
        if (sm[k]) atomicMax(mx + k, sm[k]);
}
__global__ void encode_kernel(size_t N, int nz, const float4* __restrict__ src, uint2* __restrict__ dst, int dtype,
                              const float4* __restrict__ inv_tab) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float4 v = src[i], inv = inv_tab[i % (size_t)nz];
    uint2 o;
    if (dtype == GRID_F16) {
        __half2 a = __floats2half2_rn(v.x * inv.x, v.y * inv.y), b = __floats2half2_rn(v.z * inv.z, v.w * inv.w);
        o.x = *reinterpret_cast<unsigned*>(&a); o.y = *reinterpret_cast<unsigned*>(&b);
    } else {
        __nv_bfloat162 a = __floats2bfloat162_rn(v.x * inv.x, v.y * inv.y), b = __floats2bfloat162_rn(v.z * inv.z, v.w * inv.w);
        o.x = *reinterpret_cast<unsigned*>(&a); o.y = *reinterpret_cast<unsigned*>(&b);
    }
    dst[i] = o;
}
__global__ void decode_kernel(size_t N, int nz, const uint2* __restrict__ src, float4* __restrict__ dst, int dtype,
                              const float4* __restrict__ sc_tab) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const uint2 u = src[i];
    const float4 sc = sc_tab[i % (size_t)nz];
    float2 a, b;
    if (dtype == GRID_F16) { a = __half22float2(*reinterpret_cast<const __half2*>(&u.x)); b = __half22float2(*reinterpret_cast<const __half2*>(&u.y)); }
    else { a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.x)); b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u.y)); }
    dst[i] = make_float4(a.x * sc.x, a.y * sc.y, b.x * sc.z, b.y * sc.w);
}

}  // namespace

// Per plane and channel a power-of-two scale: fp16 maps the plane's max |c| to [16384, 32768)
// (headroom below 65504, the full normal range below it), so the coefficients of every plane
// keep fp16's 11-bit relative precision however fast the channel grows towards the surface;
// bf16 has the fp32 exponent range and only needs max |c| ~ 1.
int encode_grid_16(const float4* src, void* dst, size_t nvox, int nz, int dtype, float* plane_scale_out, cudaStream_t s) {
    if (nz <= 0 || nz > 3072) return -1;             // the per-plane table lives in 48 KB of shared memory
    unsigned int* dmx = nullptr;
    float4* dinv = nullptr;
    if (cudaMalloc(&dmx, (size_t)nz * 16) != cudaSuccess) return -1;
    if (cudaMalloc(&dinv, (size_t)nz * 16) != cudaSuccess) { cudaFree(dmx); return -1; }
    cudaMemsetAsync(dmx, 0, (size_t)nz * 16, s);
    plane_absmax_kernel<<<592, 256, (size_t)nz * 16, s>>>(nvox, nz, src, dmx);
    std::vector<unsigned int> hm(4 * (size_t)nz);
    cudaMemcpyAsync(hm.data(), dmx, (size_t)nz * 16, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { cudaFree(dmx); cudaFree(dinv); return -1; }
    std::vector<float> inv(4 * (size_t)nz);
    for (size_t k = 0; k < hm.size(); k++) {
        float m;
        std::memcpy(&m, &hm[k], 4);
        float sc = 1.f;
        if (m > 0.f) sc = std::ldexp(1.0f, (int)std::ceil(std::log2((double)m)) - (dtype == GRID_F16 ? 15 : 0));
        plane_scale_out[k] = sc;
        inv[k] = 1.f / sc;
    }
    cudaMemcpyAsync(dinv, inv.data(), inv.size() * 4, cudaMemcpyHostToDevice, s);
    encode_kernel<<<(unsigned)((nvox + 255) / 256), 256, 0, s>>>(nvox, nz, src, (uint2*)dst, dtype, dinv);
    const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
    cudaFree(dmx);
    cudaFree(dinv);
    return ok ? 0 : -1;
}

int decode_grid_16(const void* src, float4* dst, size_t nvox, int nz, int dtype, const float4* d_plane_scale, cudaStream_t s) {
    decode_kernel<<<(unsigned)((nvox + 255) / 256), 256, 0, s>>>(nvox, nz, (const uint2*)src, dst, dtype, d_plane_scale);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

namespace {
__global__ void low_planes_kernel(size_t n, int nz, int nzl, const float4* __restrict__ src, float4* __restrict__ dst) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const size_t col = t / (size_t)nzl;
    const int z = (int)(t - col * (size_t)nzl);
    dst[t] = src[col * (size_t)nz + z];
}
}  // namespace

int extract_low_planes(const float4* src, size_t nxy, int nz, int nzl, float4* dst, cudaStream_t s) {
    if (nzl < 1 || nzl > nz) return -1;
    const size_t n = nxy * (size_t)nzl;
    low_planes_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, nz, nzl, src, dst);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

namespace {

// Raw (unfitted) FP64 channels of the x-planes [x0, x0 + xs): Morse (Pauli, London) and Ewald-2D,
// each xs * ny * nz values, z-fastest, into paul / lond / coul (device).
int grid_raw_channels(const GridBuildArgs& A, int x0, int xs, double* paul, double* lond, double* coul, DevBuf& buf,
                      cudaStream_t s, char* err, int errlen) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const size_t N = (size_t)xs * ny * nz;
    // host copy of ions for layer grouping and the geometry checks
    std::vector<double> hion(4 * (size_t)A.nions);
    GB_CHECK(cudaMemcpyAsync(hion.data(), A.ions, hion.size() * 8, cudaMemcpyDeviceToHost, s));
    GB_CHECK(cudaStreamSynchronize(s));
    double ztop = -1e300, qsum = 0.0, qz = 0.0;
    for (int i = 0; i < A.nions; i++) { ztop = std::max(ztop, hion[4 * i + 2]); qsum += hion[4 * i + 3]; qz += hion[4 * i + 3] * hion[4 * i + 2]; }
    const double dmin = A.p0[2] - ztop;
    if (!(dmin > 0.05)) { std::snprintf(err, errlen, "grid bottom z=%g must lie above the top ion z=%g", A.p0[2], ztop); return -1; }
    if (std::fabs(qsum) > 1e-6 * std::max(1.0, (double)A.nions)) { std::snprintf(err, errlen, "slab charge %g is not neutral", qsum); return -1; }

    // Morse channels
    {
        const float rc2 = A.morse_rcut > 0 ? (float)(A.morse_rcut * A.morse_rcut) : 3.0e38f;
        const unsigned blocks = (unsigned)((N + 127) / 128);
        morse_kernel<<<blocks, 128, 0, s>>>(A.nions, A.ions, A.ion_re, A.Lx, A.Ly, A.npbc, x0, xs, ny, nz, A.p0[0], A.p0[1], A.p0[2],
                                            A.step[0], A.step[1], A.step[2], (float)A.alpha, rc2, paul, lond);
        GB_CHECK(cudaGetLastError());
    }

    // Ewald-2D
    {
        const double g1 = 2.0 * kPi / A.Lx, g2 = 2.0 * kPi / A.Ly, area = A.Lx * A.Ly;
        const double tol = A.ewald_tol > 0 ? A.ewald_tol : 1e-12;
        const double gmax = -std::log(tol) / dmin;
        const int H = std::max(1, (int)std::floor(gmax / g1)), K = std::max(1, (int)std::floor(gmax / g2));
        const int w = 2 * H + 1, nk = 2 * K + 1;
        std::vector<double> hdz(A.nions);
        for (int i = 0; i < A.nions; i++) hdz[i] = A.p0[2] - hion[4 * i + 2];
        double* ddz;
        double2 *X, *Y, *S;
        GB_CHECK(buf.alloc(&ddz, A.nions));
        GB_CHECK(cudaMemcpyAsync(ddz, hdz.data(), A.nions * 8, cudaMemcpyHostToDevice, s));
        GB_CHECK(buf.alloc(&X, (size_t)A.nions * w)); GB_CHECK(buf.alloc(&Y, (size_t)A.nions * nk)); GB_CHECK(buf.alloc(&S, (size_t)w * nk));
        phase_table_kernel<<<(A.nions * w + 255) / 256, 256, 0, s>>>(A.nions, A.ions, 0, g1, H, X);
        phase_table_kernel<<<(A.nions * nk + 255) / 256, 256, 0, s>>>(A.nions, A.ions, 1, g2, K, Y);
        structure_factor_kernel<<<(w * nk + 127) / 128, 128, 0, s>>>(A.nions, A.ions, ddz, X, Y, H, K, g1, g2, S);
        GB_CHECK(cudaGetLastError());
        std::vector<double2> hS((size_t)w * nk);
        // the handle's stream does not synchronise with the legacy default stream: copy on it and wait
        GB_CHECK(cudaMemcpyAsync(hS.data(), S, hS.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
        GB_CHECK(cudaStreamSynchronize(s));
        // amplitudes at the grid bottom and their pruning threshold
        std::vector<double2> amp;
        std::vector<int> hcol, rowptr(1, 0), krow;
        std::vector<double> gn;
        double amax = 0.0;
        for (int kk = 0; kk < nk; kk++)
            for (int hh = 0; hh < w; hh++) {
                if (hh == H && kk == K) continue;
                const double Gx = (hh - H) * g1, Gy = (kk - K) * g2, G = std::sqrt(Gx * Gx + Gy * Gy);
                if (G > gmax) continue;
                const double2 v = hS[(size_t)kk * w + hh];
                amax = std::max(amax, (std::fabs(v.x) + std::fabs(v.y)) * 2.0 * kPi / (area * G));
            }
        const double thresh = tol * std::max(amax, 1e-300);
        for (int kk = 0; kk < nk; kk++) {
            bool any = false;
            for (int hh = 0; hh < w; hh++) {
                if (hh == H && kk == K) continue;
                const double Gx = (hh - H) * g1, Gy = (kk - K) * g2, G = std::sqrt(Gx * Gx + Gy * Gy);
                if (G > gmax) continue;
                const double2 v = hS[(size_t)kk * w + hh];
                const double pref = 2.0 * kPi / (area * G);
                if ((std::fabs(v.x) + std::fabs(v.y)) * pref < thresh) continue;
                amp.push_back(make_double2(v.x * pref, v.y * pref));
                hcol.push_back(hh - H);
                gn.push_back(G);
                any = true;
            }
            if (any) { rowptr.push_back((int)amp.size()); krow.push_back(kk - K); }
        }
        const int nrows = (int)krow.size();
        const int ne = (int)amp.size();
        // h multipliers used anywhere -> compact column index into the x phase table
        std::vector<int> hmul;
        for (int h = -H; h <= H; h++) hmul.push_back(h);
        std::vector<int> hidx(ne);
        for (int e = 0; e < ne; e++) hidx[e] = hcol[e] + H;
        int *drow, *dhidx, *dk, *dhm;
        double2 *damp, *dampz, *B, *Ex, *Ey;
        double* dgn;
        GB_CHECK(buf.alloc(&drow, rowptr.size())); GB_CHECK(buf.alloc(&dhidx, ne)); GB_CHECK(buf.alloc(&dk, nrows));
        GB_CHECK(buf.alloc(&dhm, hmul.size()));
        GB_CHECK(buf.alloc(&damp, ne)); GB_CHECK(buf.alloc(&dampz, ne)); GB_CHECK(buf.alloc(&dgn, ne));
        GB_CHECK(buf.alloc(&B, (size_t)std::max(nrows, 1) * nx));
        GB_CHECK(buf.alloc(&Ex, hmul.size() * (size_t)nx)); GB_CHECK(buf.alloc(&Ey, (size_t)std::max(nrows, 1) * ny));
        GB_CHECK(cudaMemcpyAsync(drow, rowptr.data(), rowptr.size() * 4, cudaMemcpyHostToDevice, s));
        GB_CHECK(cudaMemcpyAsync(dhm, hmul.data(), hmul.size() * 4, cudaMemcpyHostToDevice, s));
        line_phase_kernel<<<(unsigned)((hmul.size() * nx + 255) / 256), 256, 0, s>>>((int)hmul.size(), dhm, nx, A.p0[0], A.step[0], g1, Ex);
        if (ne > 0) {
            GB_CHECK(cudaMemcpyAsync(dhidx, hidx.data(), ne * 4, cudaMemcpyHostToDevice, s));
            GB_CHECK(cudaMemcpyAsync(damp, amp.data(), ne * sizeof(double2), cudaMemcpyHostToDevice, s));
            GB_CHECK(cudaMemcpyAsync(dgn, gn.data(), ne * 8, cudaMemcpyHostToDevice, s));
            GB_CHECK(cudaMemcpyAsync(dk, krow.data(), nrows * 4, cudaMemcpyHostToDevice, s));
            line_phase_kernel<<<(unsigned)(((size_t)nrows * ny + 255) / 256), 256, 0, s>>>(nrows, dk, ny, A.p0[1], A.step[1], g2, Ey);
        }
        GB_CHECK(cudaGetLastError());
        for (int iz = 0; iz < nz; iz++) {
            const double z = A.p0[2] + iz * A.step[2];
            const double phi0 = -(2.0 * kPi / area) * (qsum * z - qz);
            if (nrows > 0) {
                plane_amp_kernel<<<(ne + 255) / 256, 256, 0, s>>>(ne, damp, dgn, iz * A.step[2], thresh, dampz);
                ewald_stage1<<<(nrows * nx + 127) / 128, 128, 0, s>>>(nrows, drow, dhidx, dampz, Ex, nx, B);
            }
            ewald_stage2<<<(xs * ny + 127) / 128, 128, 0, s>>>(nrows, B, Ey, nx, ny, x0, xs, phi0, iz, nz, coul);
            GB_CHECK(cudaGetLastError());
        }
        GB_CHECK(cudaStreamSynchronize(s));
    }

    return 0;
}

// exact B-spline fit of each channel (whole grid), then pack into float4
int fit_and_pack(double* paul, double* lond, double* coul, int nx, int ny, int nz, float4* out, DevBuf& buf, cudaStream_t s,
                 char* err, int errlen) {
    const size_t N = (size_t)nx * ny * nz;
    if (fit_channel(paul, nx, ny, nz, s, buf, err, errlen)) return -1;
    if (fit_channel(lond, nx, ny, nz, s, buf, err, errlen)) return -1;
    if (fit_channel(coul, nx, ny, nz, s, buf, err, errlen)) return -1;
    pack_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(N, paul, lond, coul, out);
    GB_CHECK(cudaGetLastError());
    GB_CHECK(cudaStreamSynchronize(s));
    return 0;
}

// three channels <-> one voxel-major array of (Pauli, London, Coulomb) triples
__global__ void interleave_kernel(size_t n, const double* __restrict__ a, const double* __restrict__ b,
                                  const double* __restrict__ c, double* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { out[3 * i] = a[i]; out[3 * i + 1] = b[i]; out[3 * i + 2] = c[i]; }
}
__global__ void deinterleave_kernel(size_t n, const double* __restrict__ in, double* __restrict__ a, double* __restrict__ b,
                                    double* __restrict__ c) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { a[i] = in[3 * i]; b[i] = in[3 * i + 1]; c[i] = in[3 * i + 2]; }
}

}  // namespace

int build_grid_device(const GridBuildArgs& A, float4* out, cudaStream_t s, char* err, int errlen) {
    const size_t N = (size_t)A.nx * A.ny * A.nz;
    DevBuf buf;
    double *paul, *lond, *coul;
    GB_CHECK(buf.alloc(&paul, N)); GB_CHECK(buf.alloc(&lond, N)); GB_CHECK(buf.alloc(&coul, N));
    if (grid_raw_channels(A, 0, A.nx, paul, lond, coul, buf, s, err, errlen)) return -1;
    return fit_and_pack(paul, lond, coul, A.nx, A.ny, A.nz, out, buf, s, err, errlen);
}

int grid_raw_slab_device(const GridBuildArgs& A, int x0, int xs, double* raw, cudaStream_t s, char* err, int errlen) {
    const size_t N = (size_t)xs * A.ny * A.nz;
    DevBuf buf;
    double *paul, *lond, *coul;
    GB_CHECK(buf.alloc(&paul, N)); GB_CHECK(buf.alloc(&lond, N)); GB_CHECK(buf.alloc(&coul, N));
    if (grid_raw_channels(A, x0, xs, paul, lond, coul, buf, s, err, errlen)) return -1;
    interleave_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(N, paul, lond, coul, raw);
    GB_CHECK(cudaGetLastError());
    GB_CHECK(cudaStreamSynchronize(s));
    return 0;
}

int grid_from_raw_device(const double* raw, int nx, int ny, int nz, float4* out, cudaStream_t s, char* err, int errlen) {
    const size_t N = (size_t)nx * ny * nz;
    DevBuf buf;
    double *paul, *lond, *coul;
    GB_CHECK(buf.alloc(&paul, N)); GB_CHECK(buf.alloc(&lond, N)); GB_CHECK(buf.alloc(&coul, N));
    deinterleave_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(N, raw, paul, lond, coul);
    GB_CHECK(cudaGetLastError());
    return fit_and_pack(paul, lond, coul, nx, ny, nz, out, buf, s, err, errlen);
}

// ---- brick copy for the stencil reads of the relax kernel (layout: smr_internal.h)
namespace {
template <typename V, int DY>
__global__ void brick_kernel(const V* __restrict__ g, int nx, int ny, int nz, unsigned long long total, V* __restrict__ b) {
    const unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int e = (int)(t % (DY * 4));
    unsigned long long br = t / (DY * 4);
    const int nzb = nz - 3;
    const int jz = (int)(br % nzb); br /= nzb;
    const int iy = (int)(br % ny);
    const int ix = (int)(br / ny);
    const int dy = e >> 2, k = e & 3;
    const int y = iy + dy >= ny ? iy + dy - ny : iy + dy;
    b[t] = g[(size_t)(jz + k) + (size_t)nz * ((size_t)y + (size_t)ny * ix)];
}
}  // namespace

size_t grid_brick_bytes(int nx, int ny, int nz) {
    if (nx < 1 || ny < 4 || nz < 4) return 0;
    const unsigned long long elems = (unsigned long long)nx * ny * (nz - 3) * 8;   // float4 elements (16-bit: 16 of 8 B)
    if (elems * 2 >= (1ull << 32)) return 0;          // the kernel indexes 8-byte voxels with 32-bit offsets
    return (size_t)elems * 16;
}

int build_grid_bricks(const void* grid, int dtype, int nx, int ny, int nz, void* bricks, cudaStream_t s) {
    const size_t bytes = grid_brick_bytes(nx, ny, nz);
    if (!bytes) return (int)cudaErrorInvalidValue;
    if (dtype == GRID_F32) {
        const unsigned long long total = bytes / 16;
        brick_kernel<float4, 2><<<(unsigned)((total + 255) / 256), 256, 0, s>>>((const float4*)grid, nx, ny, nz, total, (float4*)bricks);
    } else {
        const unsigned long long total = bytes / 8;
        brick_kernel<uint2, 4><<<(unsigned)((total + 255) / 256), 256, 0, s>>>((const uint2*)grid, nx, ny, nz, total, (uint2*)bricks);
    }
    return (int)cudaGetLastError();
}

}  // namespace smr

// ============================================================================ allocation-free grid build
//
// smr_build_grid_static: the same grid as smr_build_grid for small substrates, for callers that
// cannot call cudaMalloc -- e.g. a host framework that owns all device memory through its own
// pool and forbids allocation after start-up (the reference's GPU harness forbids allocation in
// its step path).  All scratch lives
// in the file-scope array below: kStaticScratchBytes (8 MiB) held by every GPU that loads the
// library, until the process exits.  In host code the array's name is only a host-side stand-in,
// so the entry point looks up its device address with cudaGetSymbolAddress, once per device, on
// the first call made on that device (that first call should come before any stream capture).
// Every call shares the array: calls whose GPU work overlaps (different streams or threads) race.
// Nothing in it has to start at zero: each buffer is written before it is read.  Differences to
// smr_build_grid: no pruning of negligible reciprocal vectors (all G with |G| <= gmax are summed)
// and the structure factors are summed directly per ion; both agree to ~1e-12 relative.
static __device__ __align__(256) unsigned char smr_grid_static_scratch[8u << 20];

namespace smr {
namespace {

constexpr size_t kStaticScratchBytes = 8u << 20;
constexpr int kStaticMaxDevices = 64;
void* g_static_ptr[kStaticMaxDevices] = {nullptr};

__global__ void static_structure_factor(int nions, const double* __restrict__ ions, double z0, int H, int K,
                                        double g1, double g2, double2* __restrict__ S) {
    const int w = 2 * H + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= w * (2 * K + 1)) return;
    const double Gx = (t % w - H) * g1, Gy = (t / w - K) * g2, Gn = sqrt(Gx * Gx + Gy * Gy);
    double sr = 0.0, si = 0.0;
    for (int i = 0; i < nions; i++) {
        double s, c;
        sincos(-(Gx * ions[4 * i] + Gy * ions[4 * i + 1]), &s, &c);
        const double q = ions[4 * i + 3] * exp(-Gn * (z0 - ions[4 * i + 2]));
        sr += q * c; si += q * s;
    }
    S[t] = make_double2(sr, si);
}

// out[(m + half) * n + i] = exp(i m g (p0 + i st)), m in [-half, half]
__global__ void static_phase(int n, int half, double p0, double st, double g, double2* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (2 * half + 1) * n) return;
    double s, c;
    sincos((double)(t / n - half) * g * (p0 + (t % n) * st), &s, &c);
    out[t] = make_double2(c, s);
}

// B[kk * nx + ix] = sum_h pref(G) S(h, k) exp(-|G| dzp) Ex[h, ix] over 0 < |G| <= gmax
__global__ void static_stage1(int H, int K, const double2* __restrict__ S, double gmax, double g1, double g2, double area,
                              double dzp, int nx, const double2* __restrict__ Ex, double2* __restrict__ B) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (2 * K + 1) * nx) return;
    const int kk = t / nx, ix = t % nx, w = 2 * H + 1;
    const double Gy = (kk - K) * g2;
    double br = 0.0, bi = 0.0;
    for (int hh = 0; hh < w; hh++) {
        const double Gx = (hh - H) * g1, G = sqrt(Gx * Gx + Gy * Gy);
        if (G == 0.0 || G > gmax) continue;
        const double f = 2.0 * kPi / (area * G) * exp(-G * dzp);
        const double2 a = S[(size_t)kk * w + hh];
        const double2 c = Ex[(size_t)hh * nx + ix];
        br += f * (a.x * c.x - a.y * c.y);
        bi += f * (a.x * c.y + a.y * c.x);
    }
    B[t] = make_double2(br, bi);
}

// Thomas tables of the exact cubic B-spline fit for a line of n <= kStaticMaxLine points:
// cp, m of tridiag(1/6, b0 | 2/3 | bn, 1/6), and for the cyclic lines (Sherman-Morrison) the
// solved correction vector u.  Used by the host (for the scalar denominators) and by the device
// kernel that writes the tables into the static scratch.
constexpr int kStaticMaxLine = 512;
__host__ __device__ void thomas_tables(int n, double b0, double bn, double* cp, double* m) {
    const double a = 1.0 / 6.0, b = 2.0 / 3.0;
    m[0] = b0; cp[0] = a / m[0];
    for (int i = 1; i < n; i++) { const double di = (i == n - 1) ? bn : b; m[i] = di - a * cp[i - 1]; cp[i] = a / m[i]; }
}
__host__ __device__ void cyclic_u(int n, const double* cp, const double* m, double* u) {
    const double a = 1.0 / 6.0, gamma = -2.0 / 3.0;
    for (int i = 0; i < n; i++) u[i] = 0.0;
    u[0] = gamma; u[n - 1] = a;
    u[0] /= m[0];
    for (int i = 1; i < n; i++) u[i] = (u[i] - a * u[i - 1]) / m[i];
    for (int i = n - 2; i >= 0; i--) u[i] -= cp[i] * u[i + 1];
}

// One thread: the tables of the z (open), y and x (cyclic) lines into the static scratch;
// the table pointers travel by value as a kernel argument.
struct TabPtrs { double* p[8]; };
__global__ void static_fit_tables(int nz, int ny, int nx, TabPtrs t) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double a = 1.0 / 6.0, b = 2.0 / 3.0, gamma = -b;
    thomas_tables(nz, b, b, t.p[0], t.p[1]);
    thomas_tables(ny, b - gamma, b - a * a / gamma, t.p[2], t.p[3]);
    cyclic_u(ny, t.p[2], t.p[3], t.p[4]);
    thomas_tables(nx, b - gamma, b - a * a / gamma, t.p[5], t.p[6]);
    cyclic_u(nx, t.p[5], t.p[6], t.p[7]);
}

}  // namespace
}  // namespace smr

extern "C" int smr_build_grid_static(int nions, const double* ions, const double* ion_re, double Lx, double Ly,
                                     int nx, int ny, int nz, const double p0[3], const double step[3],
                                     const smr_grid_build_params_static* p, float* coef_out, void* stream,
                                     char* err, int errlen) {
    using namespace smr;
    auto fail = [&](int code, const char* msg) { if (err && errlen > 0) std::snprintf(err, errlen, "%s", msg); return code; };
    if (!ions || !ion_re || !p0 || !step || !p || !coef_out || nions <= 0) return fail(-1, "null argument or no ions");
    if (p->dtype != GRID_F32) return fail(-5, "only float32 output is supported without allocation");
    if (nx < 4 || ny < 4 || nz < 4 || nx > kStaticMaxLine || ny > kStaticMaxLine || nz > kStaticMaxLine)
        return fail(-1, "grid dimensions must be in [4, 512]");
    if (!(Lx > 0 && Ly > 0)) return fail(-1, "cell must be positive");
    double ztop = -1e300, qsum = 0.0, qz = 0.0;
    for (int i = 0; i < nions; i++) { ztop = std::max(ztop, ions[4 * i + 2]); qsum += ions[4 * i + 3]; qz += ions[4 * i + 3] * ions[4 * i + 2]; }
    const double dmin = p0[2] - ztop;
    if (!(dmin > 0.05)) return fail(-1, "grid bottom must lie above the top ion");
    if (std::fabs(qsum) > 1e-6 * std::max(1.0, (double)nions)) return fail(-1, "slab is not neutral");
    const double g1 = 2.0 * kPi / Lx, g2 = 2.0 * kPi / Ly, area = Lx * Ly;
    const double tol = p->ewald_tol > 0 ? p->ewald_tol : 1e-12;
    const double gmax = -std::log(tol) / dmin;
    // reciprocal-lattice extents, bounded before the conversion to int (a large cell or a grid
    // bottom close to the top ion gives quotients far beyond what the scratch could hold)
    const double hq = std::floor(gmax / g1), kq = std::floor(gmax / g2);
    if (!(hq <= 1e5 && kq <= 1e5)) return fail(-3, "reciprocal sum too large for the static scratch (raise ewald_tol or "
                                                   "the grid bottom above the slab)");
    const int H = std::max(1, (int)hq), K = std::max(1, (int)kq);
    const int w = 2 * H + 1, nk = 2 * K + 1;
    const size_t N = (size_t)nx * ny * nz;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t need = 3 * al(N * 8) + 2 * al((size_t)nions * 32) + al((size_t)w * nk * 16) + al((size_t)w * nx * 16) +
                        al((size_t)nk * ny * 16) + al((size_t)nk * nx * 16) + 8 * al(kStaticMaxLine * 8);
    if (need > kStaticScratchBytes) {
        char msg[200];
        std::snprintf(msg, sizeof(msg), "needs %zu bytes of scratch, more than the static %zu (reduce the grid, the ions "
                      "or raise ewald_tol)", need, kStaticScratchBytes);
        return fail(-3, msg);
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kStaticMaxDevices) return fail(-2, "no current CUDA device");
    if (!g_static_ptr[dev]) {   // first call on this device: device address of the static array
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, smr_grid_static_scratch);
        if (e != cudaSuccess || !ptr) return fail(-2, cudaGetErrorString(e));
        g_static_ptr[dev] = ptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* base = (unsigned char*)g_static_ptr[dev];
    size_t off = 0;
    auto take = [&](size_t bytes) { void* q = base + off; off += al(bytes); return q; };
    double* paul = (double*)take(N * 8);
    double* lond = (double*)take(N * 8);
    double* coul = (double*)take(N * 8);
    double* dions = (double*)take((size_t)nions * 32);
    double* dre = (double*)take((size_t)nions * 32);
    double2* S = (double2*)take((size_t)w * nk * 16);
    double2* Ex = (double2*)take((size_t)w * nx * 16);
    double2* Ey = (double2*)take((size_t)nk * ny * 16);
    double2* B = (double2*)take((size_t)nk * nx * 16);
    double* tab[8];
    for (int k = 0; k < 8; k++) tab[k] = (double*)take(kStaticMaxLine * 8);
#define ST_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) return fail(-2, cudaGetErrorString(e_)); } while (0)
    ST_CHECK(cudaMemcpyAsync(dions, ions, (size_t)nions * 32, cudaMemcpyHostToDevice, s));
    ST_CHECK(cudaMemcpy2DAsync(dre, 32, ion_re, 16, 16, nions, cudaMemcpyHostToDevice, s));
    const float rc2 = p->morse_rcut > 0 ? (float)(p->morse_rcut * p->morse_rcut) : 3.0e38f;
    morse_kernel<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(nions, dions, dre, Lx, Ly, p->npbc, 0, nx, ny, nz, p0[0], p0[1], p0[2],
                                                             step[0], step[1], step[2], (float)p->alpha_morse, rc2, paul, lond);
    static_structure_factor<<<(unsigned)(((size_t)w * nk + 127) / 128), 128, 0, s>>>(nions, dions, p0[2], H, K, g1, g2, S);
    static_phase<<<(unsigned)(((size_t)w * nx + 255) / 256), 256, 0, s>>>(nx, H, p0[0], step[0], g1, Ex);
    static_phase<<<(unsigned)(((size_t)nk * ny + 255) / 256), 256, 0, s>>>(ny, K, p0[1], step[1], g2, Ey);
    ST_CHECK(cudaGetLastError());
    for (int iz = 0; iz < nz; iz++) {
        const double z = p0[2] + iz * step[2];
        const double phi0 = -(2.0 * kPi / area) * (qsum * z - qz);
        static_stage1<<<(unsigned)(((size_t)nk * nx + 127) / 128), 128, 0, s>>>(H, K, S, gmax, g1, g2, area, iz * step[2], nx, Ex, B);
        ewald_stage2<<<(nx * ny + 127) / 128, 128, 0, s>>>(nk, B, Ey, nx, ny, 0, nx, phi0, iz, nz, coul);
    }
    ST_CHECK(cudaGetLastError());
    // exact B-spline fit: z open, y and x cyclic.  The line tables are computed on the device
    // into the scratch; the host computes only the two Sherman-Morrison denominators, from the
    // same arithmetic, and passes them by value.
    const double a = 1.0 / 6.0, b = 2.0 / 3.0, gamma = -b;
    {
        TabPtrs t;
        for (int k = 0; k < 8; k++) t.p[k] = tab[k];
        static_fit_tables<<<1, 32, 0, s>>>(nz, ny, nx, t);
        ST_CHECK(cudaGetLastError());
    }
    double den[2];
    {
        double cp[kStaticMaxLine], m[kStaticMaxLine], u[kStaticMaxLine];
        for (int axis = 0; axis < 2; axis++) {
            const int n = axis == 0 ? ny : nx;
            thomas_tables(n, b - gamma, b - a * a / gamma, cp, m);
            cyclic_u(n, cp, m, u);
            den[axis] = 1.0 + u[0] + a * u[n - 1] / gamma;
        }
    }
    for (double* ch : {paul, lond, coul}) {
        fit_z<<<(nx * ny + 127) / 128, 128, 0, s>>>(ch, nx, ny, nz, tab[0], tab[1]);
        fit_y<<<(nx * nz + 127) / 128, 128, 0, s>>>(ch, nx, ny, nz, tab[2], tab[3], tab[4], gamma, den[0]);
        fit_x<<<(ny * nz + 127) / 128, 128, 0, s>>>(ch, nx, ny, nz, tab[5], tab[6], tab[7], gamma, den[1]);
    }
    pack_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(N, paul, lond, coul, (float4*)coef_out);
    ST_CHECK(cudaGetLastError());
#undef ST_CHECK
    return 0;
}
