// ref_driver.cpp -- the reference's own OpenCL kernels, compiled for the host, behind a C ABI.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile (target `ref`) into
// oracle/_ref/libsurfref.so from the functions oracle/ref_gen.py extracts out of the
// reference's opencl/ sources.  Only tests and the fixture generator load it, to pin the
// FP64 oracle (and through it the CUDA library) to the reference's arithmetic.  Every
// kernel runs in FP32, as on an OpenCL device; NDRange and work-group sizes are those
// the reference's hosts use (32-wide groups for the NB and Morse kernels).
//
// Entry points (all arrays are the kernels' own layouts, caller-owned):
//   ref_mix_req        mixREQ_arithmetic            UFF.cl:57-65
//   ref_ljqh           getLJQH                      UFF.cl:82-95
//   ref_sample         fe3d_pbc_comb + its index tables (make_inds_pbc), in a one-line
//                      wrapper kernel that sets the tables as getNonBond_GridFF_Bspline does
//                                                    UFF.cl:1384-1511
//   ref_nb_grid        getNonBond_GridFF_Bspline    UFF.cl:1524-1718
//   ref_nb_grid_ex2    getNonBond_GridFF_Bspline_ex2 (1-2 + 1-3 exclusion list)  UFF.cl:1722-
//   ref_morse          make_MorseFF                 gridff_build.cl:217-347
//   ref_bspline_conv   BsplineConv3D                gridff_build.cl:8-61 (conv3x3_pbc GridFF.cl:539)
//   ref_ewald_coefs    compute_ewald_coefficients   Surface.cl:716-767
//   ref_ewald_full     eval_potential_full          Surface.cl:834-906
//   ref_coulomb_brute  eval_potential_brute         Surface.cl:911-954
#include "ref_cl.h"

#define DBG_UFF 0
#define IDBG_ATOM (0)
#define IDBG_SYS (0)

namespace uffcl {
#include "_ref/gen/uff.inc"
}
namespace gridcl {
#include "_ref/gen/gridff.inc"
}
namespace surfcl {
#include "_ref/gen/surface.inc"
}

namespace {

size_t round_up(size_t n, size_t m) { return (n + m - 1) / m * m; }

template <class T>
std::vector<T> padded(const T* src, size_t n, size_t total) {
    std::vector<T> v(total);
    std::memset((void*)v.data(), 0, total * sizeof(T));
    std::memcpy((void*)v.data(), (const void*)src, n * sizeof(T));
    return v;
}

float4 f4(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }
int4 i4(const int* p) { return make_int4(p[0], p[1], p[2], p[3]); }

// largest power of two <= 32 dividing n: the work-group size that leaves no partial group,
// so no work-item of make_MorseFF returns before its tile barriers
size_t group_for(size_t n) {
    size_t g = 32;
    while (g > 1 && n % g) g >>= 1;
    return g;
}

}  // namespace

extern "C" {

int ref_mix_req(int n, const float* reqi, const float* reqj, float* out) {
    for (int i = 0; i < n; i++) {
        float4 r = uffcl::mixREQ_arithmetic(f4(reqi + 4 * i), f4(reqj + 4 * i));
        std::memcpy(out + 4 * i, &r, 16);
    }
    return 0;
}

// dp (n x 3), REQij (n x 4, already mixed), R2damp -> (fx, fy, fz, E) per pair
int ref_ljqh(int n, const float* dp, const float* reqij, float R2damp, float* out) {
    for (int i = 0; i < n; i++) {
        float4 r = uffcl::getLJQH(make_float3(dp[3 * i], dp[3 * i + 1], dp[3 * i + 2]), f4(reqij + 4 * i), R2damp);
        std::memcpy(out + 4 * i, &r, 16);
    }
    return 0;
}

// u (np x 3, grid units), PLQH (np x 4), grid (nx*ny*nz float4, z fastest) -> fe3d_pbc_comb (np x 4)
int ref_sample(int np, const float* u, const float* plqh, int nx, int ny, int nz, const float* grid, float* out) {
    const size_t g[3] = {round_up((size_t)np, 32), 1, 1}, l[3] = {32, 1, 1};
    const float4* Es = reinterpret_cast<const float4*>(grid);
    clref::launch(g, l, [&]() {
        const int ip = (int)get_global_id(0), iL = (int)get_local_id(0);
        static int4 xqs[4], yqs[4];
        if (iL < 4) xqs[iL] = uffcl::make_inds_pbc(nx, iL);
        else if (iL < 8) yqs[iL - 4] = uffcl::make_inds_pbc(ny, iL - 4);
        barrier(CLK_LOCAL_MEM_FENCE);
        if (ip >= np) return;
        float4 r = uffcl::fe3d_pbc_comb(make_float3(u[3 * ip], u[3 * ip + 1], u[3 * ip + 2]), make_int3(nx, ny, nz), Es,
                                        f4(plqh + 4 * ip), xqs, yqs);
        std::memcpy(out + 4 * ip, &r, 16);
    });
    return 0;
}

// nsys systems of natoms atoms each (uniform stride, as the kernel indexes them):
// atoms / REQKs (nsys*natoms x 4), neighs / neighCell (nsys*natoms x 4), lvecs (nsys x 12),
// nPBC (4), GFFParams (4), grid (float4 coefficients) with grid_ns (4), grid_invStep (4),
// grid_p0 (4); forces (nsys*natoms x 4) are accumulated into (forces[iaa] += fe).
// nbff_on = 0 sets ns.w = -1, which skips the atom-atom part (grid only).
int ref_nb_grid(int nsys, int natoms, const float* atoms, const float* reqks, const int* neighs, const int* neighcell,
                const float* lvecs, const int* npbc, const float* gffp, const float* grid, const int* grid_ns,
                const float* grid_inv_step, const float* grid_p0, float* forces, int nbff_on) {
    const size_t nG = round_up((size_t)natoms, 32), ntot = (size_t)nsys * natoms, pad = ntot + nG;
    auto A = padded(reinterpret_cast<const float4*>(atoms), ntot, pad);
    auto R = padded(reinterpret_cast<const float4*>(reqks), ntot, pad);
    auto N = padded(reinterpret_cast<const int4*>(neighs), ntot, pad);
    auto C = padded(reinterpret_cast<const int4*>(neighcell), ntot, pad);
    auto F = padded(reinterpret_cast<const float4*>(forces), ntot, pad);
    std::vector<uffcl::cl_Mat3> lv(nsys);
    std::memcpy((void*)lv.data(), lvecs, sizeof(uffcl::cl_Mat3) * nsys);
    float4* Es = const_cast<float4*>(reinterpret_cast<const float4*>(grid));
    const size_t g[3] = {nG, (size_t)nsys, 1}, l[3] = {32, 1, 1};
    clref::launch(g, l, [&]() {
        uffcl::getNonBond_GridFF_Bspline(make_int4(natoms, 0, 0, nbff_on ? 0 : -1), A.data(), F.data(), R.data(), N.data(),
                                         C.data(), lv.data(), i4(npbc), f4(gffp), Es, i4(grid_ns), f4(grid_inv_step),
                                         f4(grid_p0));
    });
    std::memcpy(forces, F.data(), ntot * 16);
    return 0;
}

// As ref_nb_grid with the packed exclusion list excl (nsys*natoms x EXCL_MAX, sorted, -1 padded)
// in place of neighs / neighCell.
int ref_nb_grid_ex2(int nsys, int natoms, const float* atoms, const float* reqks, const int* excl, const float* lvecs,
                    const int* npbc, const float* gffp, const float* grid, const int* grid_ns, const float* grid_inv_step,
                    const float* grid_p0, float* forces) {
    const int EX = EXCL_MAX;
    const size_t nG = round_up((size_t)natoms, 32), ntot = (size_t)nsys * natoms, pad = ntot + nG;
    auto A = padded(reinterpret_cast<const float4*>(atoms), ntot, pad);
    auto R = padded(reinterpret_cast<const float4*>(reqks), ntot, pad);
    std::vector<int> X(pad * EX, -1);
    std::memcpy(X.data(), excl, ntot * EX * sizeof(int));
    auto F = padded(reinterpret_cast<const float4*>(forces), ntot, pad);
    std::vector<uffcl::cl_Mat3> lv(nsys);
    std::memcpy((void*)lv.data(), lvecs, sizeof(uffcl::cl_Mat3) * nsys);
    float4* Es = const_cast<float4*>(reinterpret_cast<const float4*>(grid));
    const size_t g[3] = {nG, (size_t)nsys, 1}, l[3] = {32, 1, 1};
    clref::launch(g, l, [&]() {
        uffcl::getNonBond_GridFF_Bspline_ex2(make_int4(natoms, 0, 0, 0), A.data(), F.data(), R.data(), X.data(), lv.data(),
                                             i4(npbc), f4(gffp), Es, i4(grid_ns), f4(grid_inv_step), f4(grid_p0));
    });
    std::memcpy(forces, F.data(), ntot * 16);
    return 0;
}

// make_MorseFF over the nGrid[0] x nGrid[1] x nGrid[2] points of the cell (x fastest):
// atoms / REQs (nAtoms x 4), nPBC (4), nGrid (4), lvec_a/b/c (4 each), grid_p0 (4),
// GFFParams (4) -> E_Paul, E_Lond (one float per point)
int ref_morse(int nAtoms, const float* atoms, const float* reqs, const int* npbc, const int* ngrid, const float* la,
              const float* lb, const float* lc, const float* p0, const float* gffp, float* e_paul, float* e_lond) {
    const size_t npts = (size_t)ngrid[0] * ngrid[1] * ngrid[2];
    const size_t grp = group_for(npts);
    const size_t na = round_up((size_t)nAtoms, 32) + 32;
    auto A = padded(reinterpret_cast<const float4*>(atoms), nAtoms, na);
    auto R = padded(reinterpret_cast<const float4*>(reqs), nAtoms, na);
    const size_t g[3] = {npts, 1, 1}, l[3] = {grp, 1, 1};
    clref::launch(g, l, [&]() {
        gridcl::make_MorseFF(nAtoms, A.data(), R.data(), e_paul, e_lond, i4(npbc), i4(ngrid), f4(la), f4(lb), f4(lc), f4(p0),
                             f4(gffp));
    });
    return 0;
}

// BsplineConv3D: Gs, G0 (nx*ny*nz, x fastest; G0 may be null) -> out = coefs.x*conv(Gs) + coefs.y*G0
int ref_bspline_conv(int nx, int ny, int nz, const float* Gs, const float* G0, float* out, float cx, float cy) {
    const size_t g[3] = {(size_t)nx, (size_t)ny, (size_t)nz}, l[3] = {1, 1, 1};
    clref::launch(g, l, [&]() { gridcl::BsplineConv3D(make_int4(nx, ny, nz, 0), Gs, G0, out, make_float2(cx, cy)); });
    return 0;
}

// compute_ewald_coefficients: ion_data (N_ions x 4: x, y, z, q), G_data (N_G x 4: h, k, |G|, -),
// b_vectors (2 x 2), area -> C_G (N_G x 2), w (N_G*N_ions x 2; may be null)
int ref_ewald_coefs(int N_ions, const float* ions, int N_G, const float* G, const float* b, float area, float* C_G, float* w) {
    const size_t g[3] = {(size_t)N_G, 1, 1}, l[3] = {1, 1, 1};
    clref::launch(g, l, [&]() {
        surfcl::compute_ewald_coefficients(reinterpret_cast<const float4*>(ions), reinterpret_cast<const float4*>(G),
                                           reinterpret_cast<const float2*>(b), area, N_ions, N_G,
                                           reinterpret_cast<float2*>(C_G), reinterpret_cast<float2*>(w));
    });
    return 0;
}

// eval_potential_full: points (N_points x 4), w, ions, G_data, b_vectors, area -> phi (N_points)
int ref_ewald_full(int N_points, const float* pts, const float* w, int N_ions, const float* ions, int N_G, const float* G,
                   const float* b, float area, float* phi) {
    const size_t g[3] = {(size_t)N_points, 1, 1}, l[3] = {1, 1, 1};
    clref::launch(g, l, [&]() {
        surfcl::eval_potential_full(reinterpret_cast<const float4*>(pts), reinterpret_cast<const float2*>(w),
                                    reinterpret_cast<const float4*>(ions), reinterpret_cast<const float4*>(G),
                                    reinterpret_cast<const float2*>(b), area, N_points, N_ions, N_G, phi);
    });
    return 0;
}

// eval_potential_brute: points (N_points x 4), ions (N_ions x 4), cell vectors a, b (2 each), N_rep -> phi
int ref_coulomb_brute(int N_points, const float* pts, int N_ions, const float* ions, const float* a, const float* b, int N_rep,
                      float* phi) {
    const size_t g[3] = {(size_t)N_points, 1, 1}, l[3] = {1, 1, 1};
    clref::launch(g, l, [&]() {
        surfcl::eval_potential_brute(reinterpret_cast<const float4*>(pts), reinterpret_cast<const float4*>(ions),
                                     reinterpret_cast<const float2*>(a), reinterpret_cast<const float2*>(b), N_points, N_ions,
                                     N_rep, phi);
    });
    return 0;
}

}  // extern "C"
