// wenofv_stage.cuh -- the fused RK-stage kernel of the WENOFV hot path (sm_100a).
//
// One launch performs one SSP-RK stage for every work item of every instance it is given:
// ghost fill (as periodic/outflow index maps on load) -> y-direction WENO sweep ->
// x-direction WENO sweep -> bound-preserving theta limiter -> Riemann fluxes at the face
// Gauss-Lobatto points -> GL quadrature -> RHS -> RK combination -> (final stage) CFL
// max-wavespeed reduction.  Nothing but the cell averages touches HBM.
//
// A work item is a strip of TX columns and a run of rows of one instance.  The CTA streams
// through the rows: iteration r loads row r+H+1 (cp.async into an 8-row ring; H = 2 for the
// 5-point WENO-JS/Z, 3 for the 7-point WENOEXP), sweeps row r in y, reconstructs the face
// states of row r in x, solves the Riemann problems of row r's x-faces and of the y-faces
// between rows r-1 and r, and updates row r-1.  The y-sweep of a column is shared by the 7
// cells whose stencils contain it (the reference recomputes it per cell,
// src/WENOFV.cpp:670-687 and :796-833, with identical operands).
//
// Thread mapping (NT threads, 128 or 256): a unit of the y-sweep is (position, variable), of the
// x-sweep (cell, variable), of the Riemann phase (face, Gauss point) and of the update
// (cell, variable); groups of NV (or 4) consecutive lanes belong to the same position, cell
// or face.  The limiter's theta and the GL quadrature sums are exchanged by warp shuffles;
// the characteristic values of a point pass between a cell's lanes through the warp's own
// shared-memory rows.  TX = NT/NV - 2(H+1) makes the y-sweep exactly one unit per thread.
#pragma once
#include "wenofv_math.cuh"

// WENOFV_CHECK_BOUNDS=1 builds the self-checking variant (lib/libwenofv_b200_checked.so):
// every global index of the stage kernel is checked against its buffer before the access,
// and a violation sets WENOFV_FLAG_BOUNDS with the cell instead of touching the memory
#ifndef WENOFV_CHECK_BOUNDS
#define WENOFV_CHECK_BOUNDS 0
#endif

namespace wenofv {
#if WENOFV_STRICT
namespace strict {
#else
namespace fast {
#endif

// Threads per CTA of a stage kernel: 128 (strips of 26 columns for the 4-variable systems)
// or, for the 4-variable systems except PRIMITIVE3 and the stiffened gas, also 256 (strips of
// 58 columns).  The wide form cuts the halo positions and idle lanes of the x-sweep, Riemann
// and update phases from ~19 % to ~9 % of the thread slots, which makes it 15 % faster on a
// 1024-wide grid (FP64: 0.892 ms per 1024^2 stage against 1.053; FP32-bulk 0.776 against
// 0.838), but a narrow grid fills its last strip poorly (a 64-wide grid runs 58 + 6 columns),
// so the engine chooses the width per instance.  PRIMITIVE3 stays at 128 (its variable-major
// y-sweep maps 4 warps to 32 positions), as does the stiffened gas (whose Newton equilibrium
// spills at 128 registers); scalar advection has strips of 122 columns at 128 already.
template <int EQ, int RECON, class R> struct StageWide {
    static constexpr bool value = EqTraits<EQ>::NV == 4 && EQ != EQ_TWO_PHASE_SG;
};
constexpr int CFL_NT = 128; // threads per CTA of cfl_kernel

// the reconstruction of one stencil at the Gauss-Lobatto points, by scheme: the 5-point
// WENO-JS/Z (half-width H = 2) or the 7-point WENOEXP (H = 3, FP64 only)
template <class R, int SCH> struct StencilRecon {
    static constexpr int H = 2, NS = 5;
    Weno5<R, SCH> W;
    __device__ __forceinline__ void init(const R *v, int scheme, int, double) { W.init(scheme, v[0], v[1], v[2], v[3], v[4]); }
    __device__ __forceinline__ void eval4(R *o) const { W.eval4(o); }
    __device__ __forceinline__ void eval03(R &o0, R &o3) const { W.eval03(o0, o3); }
};
template <class R> struct StencilRecon<R, 2> {
    static_assert(sizeof(R) == sizeof(double), "WENOEXP runs in FP64");
    static constexpr int H = 3, NS = 7;
    WenoExp W;
    __device__ __forceinline__ void init(const R *v, int, int, double dx4) { W.init(v, dx4); }
    __device__ __forceinline__ void eval4(R *o) const { W.eval4(o); }
    __device__ __forceinline__ void eval03(R &o0, R &o3) const { W.eval03(o0, o3); }
};
// PRIMITIVE3 (RECONSTRUCTIONTYPE 4, src/WENOFV.cpp:1293-1331): z1 (variable 0) through the
// WENOEXP/THINC kernel, the pressure and the velocities through WENO-Z on the middle 5
// points, whatever SCHEME is.  FP64 only.
struct Prim3Recon {
    static constexpr int H = 3, NS = 7;
    ExpThinc E;
    Weno5<double, 1> W;
    bool z;
    __device__ __forceinline__ void init(const double *v, int, int var, double dx4)
    {
        z = var == 0;
        if (z) E.init(v, dx4);
        else W.init(1, v[1], v[2], v[3], v[4], v[5]);
    }
    __device__ __forceinline__ void eval4(double *o) const
    {
        if (z) E.eval4(o);
        else W.eval4(o);
    }
    __device__ __forceinline__ void eval03(double &o0, double &o3) const
    {
        if (z) E.eval03(o0, o3);
        else W.eval03(o0, o3);
    }
};
// the per-variable reconstruction of a non-characteristic sweep
template <class R, int SCH, int RECON> struct ReconSel { using type = StencilRecon<R, SCH>; };
template <class R, int SCH> struct ReconSel<R, SCH, 4> {
    static_assert(SCH == 2 && sizeof(R) == sizeof(double), "PRIMITIVE3 runs in FP64 on the 7-point geometry");
    using type = Prim3Recon;
};

// walls (NEUMANN 1, NOSLIP 2, FREESLIP 4): the mirror image across the boundary, reflected
// again for grids narrower than the halo; flips counts the reflections (bounded: each one
// lands at least one cell nearer to [0, n))
__device__ __forceinline__ int mirror_index(int k, int n, int &flips)
{
    flips = 0;
    for (int it = 0; it < 64 && (k < 0 || k >= n); it++) {
        k = k < 0 ? -1 - k : 2 * n - 1 - k;
        flips++;
    }
    return k < 0 ? 0 : (k >= n ? n - 1 : k);
}
__device__ __forceinline__ bool is_wall(int bc) { return bc == 1 || bc == 2 || bc == 4; }

__device__ __forceinline__ int map_index(int k, int n, int bc)
{
    if (bc == 5) return k < 0 ? 0 : (k >= n ? n - 1 : k); // outflow: zero-gradient copy
    if (is_wall(bc)) {
        int f;
        return mirror_index(k, n, f);
    }
    k %= n;
    return k < 0 ? k + n : k; // periodic wrap (2-D, corners included)
}

// the sign of variable v in a wall ghost cell reflected fx times in x and fy times in y:
// the normal momentum changes sign at each reflection, the tangential one too for NOSLIP
template <int EQ> __device__ __forceinline__ double wall_sign(int v, int fx, int fy, int bc)
{
    constexpr int MX = EQ == EQ_EULER ? 1 : 2, MY = MX + 1; // momentum components
    if (EQ == EQ_LINEAR_ADV) return 1.0;
    int n = 0;
    if (v == MX) n = fx + (bc == 2 ? fy : 0);
    else if (v == MY) n = fy + (bc == 2 ? fx : 0);
    return (n & 1) ? -1.0 : 1.0;
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void flag_error(InstState *st, unsigned int f, long long cell)
{
    atomicOr(&st->flags, f);
    atomicCAS((unsigned long long *)&st->bad_cell, (unsigned long long)-1LL, (unsigned long long)cell);
}

// finalize one instance after its final stage (or after the initial CFL pass): the
// bookkeeping of CWENOFV::run's loop, src/WENOFV.cpp:323-332
__device__ __forceinline__ void finalize_instance(InstState *st, int fin_kind, int out_buf)
{
    if (st->done) return;
    const double dtcfl = __longlong_as_double((long long)st->accum);
    st->accum = (unsigned long long)__double_as_longlong(1.0); // calculateDeltaT starts from 1.0 (:477)
    st->dtcfl = dtcfl;
    if (fin_kind == FIN_STEP) st->cur_buf = out_buf;
    if (st->mode != MODE_ADVANCE) return;
    if (fin_kind == FIN_STEP) {
        st->now += st->dt;
        st->nsteps++;
    }
    if (st->flags & 1u) { st->done = 1; return; } // NaN time step: stop (the reference aborts)
    if (fabs(st->now - st->t_end) <= 1e-10 || (st->max_steps > 0 && st->nsteps >= st->max_steps)) {
        st->done = 1;
        return;
    }
    const double remaining = st->t_end - st->now;
    st->dt = (remaining < dtcfl) ? remaining : dtcfl; // std::min(timestep, remainingTime)
}

// last-CTA-done pattern: the CTA that finishes last finalizes the launch's instances
__device__ __forceinline__ void launch_epilogue(const StageLaunch &L, int fin_kind, int *s_last)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(L.counter, 1u);
        *s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (*s_last) {
        __threadfence();
        const int nfin = L.counts ? L.counts[1] : L.nfin;
        for (int k = threadIdx.x; k < nfin; k += blockDim.x) finalize_instance(&L.state[L.fin_ids[k]], fin_kind, L.bout);
        __syncthreads();
        if (threadIdx.x == 0) *L.counter = 0u;
    }
}

__device__ __forceinline__ void cfl_atomic_min(InstState *st, double v)
{
    if (v >= 0.0) atomicMin(&st->accum, (unsigned long long)__double_as_longlong(v));
}

// block-wide minimum of a non-negative double (+inf for idle threads)
__device__ __forceinline__ double block_min(double v, double *s_red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s_red[w] = v;
    __syncthreads();
    double m = s_red[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) m = fmin(m, s_red[k]);
    return m;
}

// strip geometry for stencil half-width H: a cell's face states need the y-sweep at the
// H positions on each side of it and its neighbours', so the strip carries GH = H + 1
// halo positions on each side (GH = 3 is the reference's ghost layer count,
// src/WENOFV.cpp:59)
template <int EQ, int H, int NT> struct StageGeom {
    static constexpr int NV = EqTraits<EQ>::NV;
    static constexpr int GH = H + 1;
    static constexpr int TX = NT / NV - 2 * GH; // interior columns per strip
    static constexpr int P = TX + 2 * GH;       // y-sweep positions per row
};

// shared memory of one CTA (doubles)
template <int EQ, int H, int NT> struct StageSmem {
    static constexpr int NV = StageGeom<EQ, H, NT>::NV, TX = StageGeom<EQ, H, NT>::TX, P = StageGeom<EQ, H, NT>::P;
    // Strides are padded so that the lanes of a half-warp (8-byte accesses are served 16
    // lanes at a time) hit distinct bank pairs: rows of 4 variables at P+4 doubles
    // (variable v of 4 neighbouring positions: banks 8v + 2p), positions and cells at an odd
    // number of doubles (neighbouring positions 2 banks apart).
    static constexpr int PS = NV > 1 ? P + 4 : P; // row stride of su / sun
    static constexpr int YS = NV == 4 ? 20 : 4 * NV + 1; // position stride of sy (see sy_index)
    // face states of 4 variables: strides of 4 (mod 16) doubles with the variable slot rotated
    // by the face index (face_slot), so that both the writers (4 cells x 4 variables of a
    // half-warp, one point) and the readers (4 faces x 4 points, one variable) hit 16
    // distinct banks
    static constexpr int FS = NV == 4 ? 36 : 8 * NV + 1; // face stride of sxf
    static constexpr int BS = NV == 4 ? 20 : 4 * NV + 1; // cell stride of syb / syt
    double su[8][NV][PS];   // ring of stage-input rows
    double sun[2][NV][PS];  // U^n rows (stages after the first)
    double sy[P * YS];      // y-sweep of the current row by (position, y GL point, variable): sy_index
    double sxf[TX + 1][FS]; // x-face states: [face][(minus/plus side * 4 + GL point) * NV + var]
    double syb[TX][BS];     // bottom face states of the current row: [cell][GL point * NV + var]
    double syt[2][TX][BS];  // top face states of the current and previous row
    double sfx[2][TX + 1][NV];    // x-face quadrature sums of two rows
    double sfy[2][TX][NV];        // y-face quadrature sums below the current and previous row
    static constexpr int PE = NV > 1 ? P : 1;
    typename CellEigen<EQ>::type se[PE]; // per-cell eigensystem data of one row, by position
    double smu[PE][2];                   // the limiter's wave-speed weights mu1, mu2 by position
    double sdxc[TX], sdxl[TX];    // column widths of the strip
    double sidxc[TX], sidxl[TX];  // their reciprocals (contracted build)
    double sred[NT / 32];
    int s_last;
};

// slot of variable v in the face-state records of face (or cell) f: rotated by f for 4
// variables (the bank layout of StageSmem::FS / BS), the variable itself otherwise
template <int NV> __device__ __forceinline__ int face_slot(int v, int f)
{
    if constexpr (NV == 4) return (v + f) & 3;
    else return v;
}

// element (position p, y Gauss point g, variable v) of StageSmem::sy.  Conservative and
// characteristic sweeps (4 variables): position stride 20 (4 mod 16 doubles), so that the
// writers and the x-sweep's readers, 4 positions x 4 variables of a half-warp each, hit 16
// distinct banks; primitive sweeps (whose x-sweep lanes read one point of 4 variables per
// cell, 4 cells x 4 points) stride 4 NV + 1.
template <int RECON, int NV> __device__ __forceinline__ int sy_index(int p, int g, int v)
{
    if constexpr (NV == 4 && RECON < 2) return p * 20 + g * 4 + v;
    else return p * (4 * NV + 1) + g * NV + v;
}

// the 4 values at q (16-byte aligned) by 16-byte shared-memory loads
template <class R> __device__ __forceinline__ void load4(const R *q, R *o)
{
    if constexpr (sizeof(R) == sizeof(double)) {
        const double2 a = reinterpret_cast<const double2 *>(q)[0], b = reinterpret_cast<const double2 *>(q)[1];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    } else {
        const float4 a = reinterpret_cast<const float4 *>(q)[0];
        o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = a.w;
    }
}

// bytes of a CTA's StageSmem, rounded to 16 (the primitive ring follows it)
template <int EQ, int H, int NT> struct StageSmemBytes {
    static constexpr int value = (int)((sizeof(StageSmem<EQ, H, NT>) + 15) / 16 * 16);
};

// periodic wrap or outflow clamp (the ghost fill of the non-wall kinds)
__device__ __forceinline__ int map_index_po(int k, int n, int bc)
{
    if (bc == 5) return k < 0 ? 0 : (k >= n ? n - 1 : k);
    k %= n;
    return k < 0 ? k + n : k;
}

// the wall form of load_row: ghost cells are plain loads with the momentum signs
template <int EQ, int H, int NT>
__device__ __forceinline__ void load_row_walls(double (*dst)[StageSmem<EQ, H, NT>::PS], const double *buf, const InstDesc &D, int row,
                                            int i0, InstState *st)
{
    constexpr int P = StageGeom<EQ, H, NT>::P, NV = StageGeom<EQ, H, NT>::NV, GH = StageGeom<EQ, H, NT>::GH;
    const size_t plane = (size_t)D.ny * D.pitch;
    (void)st;
    int fy;
    const int jj = mirror_index(row, D.ny, fy);
    for (int e = threadIdx.x; e < NV * P; e += NT) {
        const int v = e / P, p = e - v * P;
        int fx;
        const int ii = mirror_index(i0 - GH + p, D.nx, fx);
#if WENOFV_CHECK_BOUNDS
        if (jj < 0 || jj >= D.ny || ii < 0 || ii >= D.nx) {
            flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)row * D.nx + (i0 - GH + p));
            continue;
        }
#endif
        if (fx | fy) dst[v][p] = wall_sign<EQ>(v, fx, fy, D.bc) * buf[v * plane + (size_t)jj * D.pitch + ii];
        else cp_async8(&dst[v][p], buf + v * plane + (size_t)jj * D.pitch + ii);
    }
}

// the NEUMANN2 form of load_row: interior cells stream in by cp.async, ghost cells are plain
// loads of the instance's fixed frame [v][ny+8][nx+8] (interior at (4, 4)).  Rows stay in
// [-GH, ny+GH) with GH <= 4; columns past nx+4 only occur in a strip's unused tail and are
// clamped into the frame.
template <int EQ, int H, int NT>
__device__ __forceinline__ void load_row_frame(double (*dst)[StageSmem<EQ, H, NT>::PS], const double *buf, const InstDesc &D, int row,
                                            int i0, InstState *st)
{
    constexpr int P = StageGeom<EQ, H, NT>::P, NV = StageGeom<EQ, H, NT>::NV, GH = StageGeom<EQ, H, NT>::GH;
    static_assert(GH <= 4, "the frame holds 4 ghost layers");
    const size_t plane = (size_t)D.ny * D.pitch;
    const int fw = D.nx + 8;
    const size_t fplane = (size_t)(D.ny + 8) * fw;
    const int fr = min(max(row, -4), D.ny + 3) + 4;
    const bool ghost_row = row < 0 || row >= D.ny;
    (void)st;
    for (int e = threadIdx.x; e < NV * P; e += NT) {
        const int v = e / P, p = e - v * P;
        const int col = i0 - GH + p;
        if (ghost_row || col < 0 || col >= D.nx) {
            const int fc = min(max(col, -4), D.nx + 3) + 4;
#if WENOFV_CHECK_BOUNDS
            if (row < -4 || row >= D.ny + 4 || col < -4) { // the clamps above only hide a strip's tail
                flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)row * D.nx + col);
                continue;
            }
#endif
            dst[v][p] = D.frame[v * fplane + (size_t)fr * fw + fc];
        } else {
            cp_async8(&dst[v][p], buf + v * plane + (size_t)row * D.pitch + col);
        }
    }
}

// the two ghost rules that are not an index map (walls, NEUMANN2 frame), behind one out-of-line
// call so that the periodic and outflow loads keep the stage kernel's register allocation
template <int EQ, int H, int NT>
__device__ __noinline__ void load_row_other(double (*dst)[StageSmem<EQ, H, NT>::PS], const double *buf, const InstDesc &D, int row,
                                            int i0, InstState *st)
{
    if (D.bc == 3) load_row_frame<EQ, H, NT>(dst, buf, D, row, i0, st);
    else load_row_walls<EQ, H, NT>(dst, buf, D, row, i0, st);
}

// one row of NV x P stage values into shared memory (ghost fill = index map), cp.async 8 B
template <int EQ, int H, int NT>
__device__ __forceinline__ void load_row(double (*dst)[StageSmem<EQ, H, NT>::PS], const double *buf, const InstDesc &D, int row,
                                         int i0, InstState *st)
{
    constexpr int P = StageGeom<EQ, H, NT>::P, NV = StageGeom<EQ, H, NT>::NV, GH = StageGeom<EQ, H, NT>::GH;
    const size_t plane = (size_t)D.ny * D.pitch;
    (void)st;
    if (D.bc == 0 || D.bc == 5) {
        const int jj = map_index_po(row, D.ny, D.bc);
#pragma unroll
        for (int e = threadIdx.x; e < NV * P; e += NT) {
            const int v = e / P, p = e - v * P;
            const int ii = map_index_po(i0 - GH + p, D.nx, D.bc);
#if WENOFV_CHECK_BOUNDS
            if (jj < 0 || jj >= D.ny || ii < 0 || ii >= D.nx) { // record and skip the access
                flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)row * D.nx + (i0 - GH + p));
                continue;
            }
#endif
            cp_async8(&dst[v][p], buf + v * plane + (size_t)jj * D.pitch + ii);
        }
        return;
    }
    load_row_other<EQ, H, NT>(dst, buf, D, row, i0, st);
}

// value of a reconstruction: in the deviation form the anchor plus the FP32 deviation, in
// FP64 the reconstructed value itself (unchanged, so the FP64 forms keep their bits)
template <bool DEV, class R> __device__ __forceinline__ double anchor(double c, R d)
{
    if constexpr (DEV) return c + (double)d;
    else return (double)d;
}

// ---- phase 0: the per-cell eigensystem data (L/R rows, wave speeds) of row r at the
// strip's P positions, computed once per cell by one thread each (threads t0 .. t0+n-1)
// instead of by every lane that needs it.  Identical arithmetic to the per-lane form.
template <int EQ, int RECON, int H, int NT>
__device__ __forceinline__ void phase_eigen(StageSmem<EQ, H, NT> &S, const InstDesc &D, int r, int t0, int n)
{
    constexpr int NV = StageGeom<EQ, H, NT>::NV, P = StageGeom<EQ, H, NT>::P;
    if constexpr (NV > 1) {
        if (!(RECON == 1 || D.limiter)) return;
        for (int p = (int)threadIdx.x - t0; p < P; p += n) {
            double u[NV];
#pragma unroll
            for (int j = 0; j < NV; j++) u[j] = S.su[r & 7][j][p];
            cell_eigen<EQ>(D.eq, u, S.se[p]);
            if (D.limiter) { // src/WENOFV.cpp:1954-1957
                double a1, a2;
                max_eigs_of<EQ>(S.se[p], a1, a2);
#if WENOFV_STRICT
                S.smu[p][0] = (a1 / D.dX) / (a1 / D.dX + a2 / D.dY);
                S.smu[p][1] = (a2 / D.dY) / (a1 / D.dX + a2 / D.dY);
#else
                // the same weights multiplied through by dX dY: one division
                const double s1 = a1 * D.dY, s2 = a2 * D.dX, iv = 1.0 / (s1 + s2);
                S.smu[p][0] = s1 * iv;
                S.smu[p][1] = s2 * iv;
#endif
            }
        }
    }
}

// ---- phase 1: y-direction sweep of row r (src/WENOFV.cpp:670-687, :796-833) ------------
// FP64: the reference's arithmetic on the averages.  FP32 bulk: the same reconstruction on
// the deviations from the column's centre average (WENO is translation invariant), so that
// FP32 rounds the small differences, not the large averages; the result is re-anchored in
// FP64.
// bytes of dynamic shared memory of a stage kernel: the primitive-variable ring of the
// primitive reconstructions (8 rows of the 4 primitives at the strip's positions)
template <int EQ, int RECON, int H, int NT> struct StageDynSmem {
    static constexpr int value = (RECON >= 2 && EqTraits<EQ>::NV == 4) ? 8 * 4 * StageSmem<EQ, H, NT>::PS * (int)sizeof(double) : 0;
};

template <int EQ, int RECON, class R, int SCH, int NT>
__device__ __forceinline__ void phase_ysweep(StageSmem<EQ, StencilRecon<R, SCH>::H, NT> &S, const InstDesc &D, int r, double *ring_raw,
                                             bool first)
{
    using SR = typename ReconSel<R, SCH, RECON>::type;
    constexpr int H = SR::H, NS = SR::NS;
    constexpr int NV = StageGeom<EQ, H, NT>::NV;
    constexpr bool DEV = sizeof(R) < sizeof(double); // deviation form
    const int t = threadIdx.x;
    // PRIMITIVE3 reconstructs z1 with another kernel than p, u, v: one warp per variable (the
    // strip's 32 positions on its lanes, the z1 warp rotating with the row) instead of the 4
    // variables of a position on 4 lanes, so that the two kernels do not diverge in a warp
    const int p = RECON == 4 ? (t & 31) + 32 * (t >> 7) : t / NV; // PRIMITIVE3: warps 4-7 take positions 32-63
    const int v = RECON == 4 ? (((t >> 5) + r) & 3) : t - p * NV;
    static_assert(RECON != 4 || (NV == 4 && StageGeom<EQ, H, NT>::P == NT / 4), "variable-major y-sweep");
    if (RECON != 1 || NV == 1) {
        // conservative: the averages; primitive (RECONSTRUCTIONTYPE 2-4): the primitive
        // variables of each of the NS cells (src/WENOFV.cpp:944-979).  Each (position,
        // variable) thread keeps the primitive values of its own column in a ring of 8 rows
        // (only it reads and writes its entries), so a row is converted once, when it enters
        // the stencil (all NS rows at the first row of a work item).
        double st[NS];
#pragma unroll
        for (int m = 0; m < NS; m++) {
            if constexpr (RECON >= 2 && NV == 4) {
                auto ring = reinterpret_cast<double (*)[4][StageSmem<EQ, H, NT>::PS]>(ring_raw);
                const int row = r - H + m;
                if (first || m == NS - 1) {
                    double U4[4], W4[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) U4[j] = S.su[row & 7][j][p];
                    tp_to_primitive(D.eq, RECON, U4, W4);
                    st[m] = W4[v];
                    ring[row & 7][v][p] = st[m];
                } else {
                    st[m] = ring[row & 7][v][p];
                }
            } else {
                (void)ring_raw; (void)first;
                st[m] = S.su[(r - H + m) & 7][v][p];
            }
        }
        const double c0 = DEV ? st[H] : 0.0;
        R sv[NS];
#pragma unroll
        for (int m = 0; m < NS; m++) sv[m] = (R)(st[m] - c0);
        SR W;
        W.init(sv, D.scheme, v, D.dx4);
        R o[4];
        W.eval4(o);
#pragma unroll
        for (int gp = 0; gp < 4; gp++) S.sy[sy_index<RECON, NV>(p, gp, v)] = anchor<DEV>(c0, o[gp]);
    } else {
        // characteristic: project with L(U_centre, y), reconstruct, project back with R(U_centre, y).
        // The eigenvectors and the forward projection are FP64 in every form: the two-phase
        // eigenvector matrices reach condition numbers of ~5e3 near pure phases, so FP32 rows
        // of L against FP32 rows of R (|R L - I| ~ 3e-4) would mix the large partial density
        // into the small momenta.
        double Uc[NV], Lrow[NV], Rrow[NV];
        R pr[NS];
#pragma unroll
        for (int j = 0; j < NV; j++) Uc[j] = S.su[r & 7][j][p];
        eigen_rows_of<EQ>(D.eq, S.se[p], false, v, Lrow, Rrow);
        // deviation form: L (U_m - Uc) = L U_m - L Uc, with L Uc formed once (FP64 keeps the
        // difference exact to ~1e-16 of the projected values, far below FP32's 6e-8)
        double lc = 0.0;
        if constexpr (DEV) {
#pragma unroll
            for (int j = 0; j < NV; j++) lc += Lrow[j] * Uc[j];
        }
#pragma unroll
        for (int m = 0; m < NS; m++) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < NV; j++) s += Lrow[j] * S.su[(r - H + m) & 7][j][p];
            pr[m] = DEV ? (R)(s - lc) : (R)s;
        }
        SR W;
        W.init(pr, D.scheme, v, D.dx4);
        R cg[4];
        W.eval4(cg);
        if constexpr (NV == 4) { // the characteristic sweeps have 4 variables
            // the 4 characteristic values of a point reach the position's 4 lanes through the
            // warp's own rows of sy (positions 8w .. 8w+7, written by no other warp), as R at the
            // element offsets of sy_index; the results overwrite them afterwards
            R *xs = reinterpret_cast<R *>(&S.sy[sy_index<RECON, NV>(p, 0, 0)]);
#pragma unroll
            for (int gp = 0; gp < 4; gp++) xs[gp * 4 + v] = cg[gp];
            __syncwarp();
            double out[4];
#pragma unroll
            for (int gp = 0; gp < 4; gp++) {
                R q[4];
                load4<R>(xs + gp * 4, q);
                // back-projection: FP32 in the bulk form (it adds an error of the same order as
                // the FP32 WENO's own, eps * sum_k |R_vk w_k|), FP64 otherwise
                if constexpr (DEV) {
                    R s = R(0);
#pragma unroll
                    for (int k = 0; k < NV; k++) s += (R)Rrow[k] * q[k];
                    out[gp] = Uc[v] + (double)s;
                } else {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < NV; k++) s += Rrow[k] * (double)q[k];
                    out[gp] = s;
                }
            }
            __syncwarp();
#pragma unroll
            for (int gp = 0; gp < 4; gp++) S.sy[sy_index<RECON, NV>(p, gp, v)] = out[gp];
        }
    }
}

// ---- phase 2: x-direction sweep + limiter of row r (src/WENOFV.cpp:690-721, :836-880,
//      limiter :1895-2000) -> face states (FP64 in every form) ------------------------------
template <int EQ, int RECON, class R, int SCH, int NT>
__device__ __forceinline__ void phase_xsweep(StageSmem<EQ, StencilRecon<R, SCH>::H, NT> &S, const InstDesc &D, InstState *st, int r,
                                             int i0, int TXe, const double *ring_raw, bool flag_row)
{
    using SR = typename ReconSel<R, SCH, RECON>::type;
    constexpr int H = SR::H, NS = SR::NS;
    constexpr int NV = StageGeom<EQ, H, NT>::NV, TX = StageGeom<EQ, H, NT>::TX, GH = StageGeom<EQ, H, NT>::GH;
    constexpr bool DEV = sizeof(R) < sizeof(double);
    const int t = threadIdx.x;
    const int cu = t / NV, v = t - cu * NV;
    const bool active = cu < TX + 2;
    const int c = (active ? cu : TX + 1) - 1; // cell in [-1, TX]
    const int lane = t & 31, gbase = lane & ~(NV - 1);
    double fv[4][4]; // face values [gpi][gpj] of variable v (boundary points only)

    if constexpr (RECON >= 2 && NV == 4) {
        // primitive reconstructions (src/WENOFV.cpp:981-1025, :1137-1189, :1302-1354): lane v
        // of the cell reconstructs all 4 primitive variables at y Gauss point gj = v, so that
        // PRIMITIVE3's z1 kernel and WENO-Z do not diverge across the cell's lanes, converts
        // its points back to conserved variables, and hands every lane its variable at the 12
        // boundary points through shared memory (below).  Lanes 1 and 2 also evaluate the
        // inner points (unused) to keep the lanes converged.
        auto ring = reinterpret_cast<const double (*)[4][StageSmem<EQ, H, NT>::PS]>(ring_raw);
        const int gj = v;
        double pv[4][4]; // [gpi][variable] at (gpi, gj)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const double ck = DEV ? ring[r & 7][k][c + GH] : 0.0; // deviation anchor: the primitive average
            R sv[NS];
#pragma unroll
            for (int m = 0; m < NS; m++) sv[m] = (R)(S.sy[sy_index<RECON, NV>(c + 1 + m, gj, k)] - ck);
            SR W;
            W.init(sv, D.scheme, k, D.dx4);
            R o[4];
            W.eval4(o);
#pragma unroll
            for (int gpi = 0; gpi < 4; gpi++) pv[gpi][k] = anchor<DEV>(ck, o[gpi]);
        }
#pragma unroll
        for (int gpi = 0; gpi < 4; gpi++) {
            double U4[4];
            tp_from_primitive(D.eq, RECON, pv[gpi], U4);
#pragma unroll
            for (int k = 0; k < 4; k++) pv[gpi][k] = U4[k];
        }
        // each lane's variable at the boundary points, through this warp's faces 8w .. 8w+6 of
        // sxf (as in the characteristic sweep): per x point gpi, lane gj leaves its 4 variables
        // at slot k*4 + ((gj + k) & 3) of its cell, so that the writers (4 cells x 4 points, one
        // variable) and the readers (4 cells x 4 variables, one point) hit 16 distinct banks
        double *xs = reinterpret_cast<double *>(&S.sxf[8 * (t >> 5)][0]) + (active ? (lane >> 2) : 0) * 20;
#pragma unroll
        for (int gpi = 0; gpi < 4; gpi++) {
            __syncwarp(); // the previous point's reads are done
            if (active) {
#pragma unroll
                for (int k = 0; k < 4; k++) xs[k * 4 + ((gj + k) & 3)] = pv[gpi][k];
            }
            __syncwarp();
#pragma unroll
            for (int gpj = 0; gpj < 4; gpj++) {
                if (!(gpi == 0 || gpi == 3 || gpj == 0 || gpj == 3)) continue;
                fv[gpi][gpj] = xs[v * 4 + ((gpj + v) & 3)];
            }
        }
        __syncwarp(); // the exchange area is written below
    } else if (RECON != 1 || NV == 1) {
        (void)ring_raw;
        double cc = 0.0; // deviation anchor: the cell's own average
        if constexpr (DEV) cc = S.su[r & 7][v][c + GH];
#pragma unroll
        for (int gpj = 0; gpj < 4; gpj++) {
            // the stencil of cell c: positions c+GH-H .. c+GH+H = c+1 .. c+1+2H
            R sv[NS];
#pragma unroll
            for (int m = 0; m < NS; m++) sv[m] = (R)(S.sy[sy_index<RECON, NV>(c + 1 + m, gpj, v)] - cc);
            SR W;
            W.init(sv, D.scheme, v, D.dx4);
            if (gpj == 0 || gpj == 3) {
                R o[4];
                W.eval4(o);
#pragma unroll
                for (int gpi = 0; gpi < 4; gpi++) fv[gpi][gpj] = anchor<DEV>(cc, o[gpi]);
            } else {
                R o0, o3;
                W.eval03(o0, o3);
                fv[0][gpj] = anchor<DEV>(cc, o0);
                fv[3][gpj] = anchor<DEV>(cc, o3);
            }
        }
    } else {
        double Uc[NV], Lrow[NV], Rrow[NV]; // FP64 in every form, as in the y-sweep
#pragma unroll
        for (int j = 0; j < NV; j++) Uc[j] = S.su[r & 7][j][c + GH];
        eigen_rows_of<EQ>(D.eq, S.se[c + GH], true, v, Lrow, Rrow);
        double lc = 0.0; // L Uc of the deviation form, as in the y-sweep
        if constexpr (DEV) {
#pragma unroll
            for (int j = 0; j < NV; j++) lc += Lrow[j] * Uc[j];
        }
        // exchange area of this warp's cells (inactive lanes read cell slot 0): element stride
        // 20 per cell (4 mod 16 doubles: the 16 writers of a half-warp hit distinct banks)
        R *xs = reinterpret_cast<R *>(&S.sxf[8 * (t >> 5)][0]) + (active ? (lane >> 2) : 0) * 20;
        // per y Gauss point: project, reconstruct, and project back at once, so that only
        // that point's characteristic values are live (not all twelve)
#pragma unroll
        for (int gpj = 0; gpj < 4; gpj++) {
            R pr[NS];
#pragma unroll
            for (int m = 0; m < NS; m++) {
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < NV; j++) s += Lrow[j] * S.sy[sy_index<RECON, NV>(c + 1 + m, gpj, j)];
                pr[m] = DEV ? (R)(s - lc) : (R)s;
            }
            SR W;
            W.init(pr, D.scheme, v, D.dx4);
            R cg[4];
            const bool all4 = gpj == 0 || gpj == 3;
            if (all4) W.eval4(cg);
            else W.eval03(cg[0], cg[3]);
            if constexpr (NV == 4) { // the characteristic sweeps have 4 variables
                // the cell's 4 characteristic values of a point through this warp's faces
                // 8w .. 8w+6 of sxf: only this warp writes them (at the end of this phase), and
                // the previous row's face states there were read before the last barrier
                __syncwarp(); // the previous point's reads are done
                if (active) {
#pragma unroll
                    for (int gpi = 0; gpi < 4; gpi++)
                        if (gpi == 0 || gpi == 3 || all4) xs[gpi * 4 + v] = cg[gpi];
                }
                __syncwarp();
#pragma unroll
                for (int gpi = 0; gpi < 4; gpi++) {
                    if (!(gpi == 0 || gpi == 3 || all4)) continue;
                    R q[4];
                    load4<R>(xs + gpi * 4, q);
                    if constexpr (DEV) { // as in the y-sweep
                        R s = R(0);
#pragma unroll
                        for (int k = 0; k < NV; k++) s += (R)Rrow[k] * q[k];
                        fv[gpi][gpj] = Uc[v] + (double)s;
                    } else {
                        double s = 0.0;
#pragma unroll
                        for (int k = 0; k < NV; k++) s += Rrow[k] * (double)q[k];
                        fv[gpi][gpj] = s;
                    }
                }
            }
        }
        __syncwarp(); // the exchange area is written below
    }

    // bound-preserving limiter: theta from the partial densities, in FP64 in every form
    constexpr int NLIM = LimitedVars<EQ>::N;
    if (NLIM > 0 && D.limiter) {
        double ub[NV];
#pragma unroll
        for (int j = 0; j < NV; j++) ub[j] = S.su[r & 7][j][c + GH];
        const double mu1 = S.smu[c + GH][0], mu2 = S.smu[c + GH][1];
        double th = 1.0;
        if (v < NLIM) {
            const double uave = ub[v];
            const double zeps = 1e-12, omega1 = 0.1, omegaR = 1.0 - 2 * omega1;
            const double eps = std_min(zeps, uave);
            double rem = uave;
#pragma unroll
            for (int gp = 0; gp < 4; gp++) {
                const double w = gl_weight(gp);
                rem -= omega1 * w / 2 * mu2 * fv[gp][0];
                rem -= omega1 * w / 2 * mu2 * fv[gp][3];
                rem -= omega1 * w / 2 * mu1 * fv[0][gp];
                rem -= omega1 * w / 2 * mu1 * fv[3][gp];
            }
#if WENOFV_STRICT
            rem /= omegaR;
#else
            rem *= 1.0 / omegaR; // a constant
#endif
            double mloc = rem;
#pragma unroll
            for (int gp = 0; gp < 4; gp++) {
                mloc = sc_min(mloc, fv[gp][0]);
                mloc = sc_min(mloc, fv[gp][3]);
                mloc = sc_min(mloc, fv[0][gp]);
                mloc = sc_min(mloc, fv[3][gp]);
            }
            th = sc_min(fabs((uave - eps) / (uave - mloc)), th);
        }
        const double t0 = __shfl_sync(0xffffffffu, th, gbase + 0);
        const double t1 = __shfl_sync(0xffffffffu, th, gbase + (NLIM > 1 ? 1 : 0));
        const double theta = NLIM == 2 ? sc_min(t0, t1) : t0;
        // the per-cell record of useBoundPreservingLimiter (src/WENOFV.cpp:1906-1909), kept
        // from the final stage of a step for the average_*.plt theta column
        if (flag_row && active && v == 0 && c >= 0 && c < TXe) {
#if WENOFV_CHECK_BOUNDS
            if (r < 0 || r >= D.ny || i0 + c >= D.nx) flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)r * D.nx + i0 + c);
            else
#endif
                D.theta_flag[(size_t)r * D.nx + i0 + c] = theta < 1.0 - 1e-8 ? 1 : 0;
        }
        if (theta >= 0.0 && theta <= 1.0) {
            const double u0 = ub[v];
#pragma unroll
            for (int gpj = 0; gpj < 4; gpj++)
#pragma unroll
                for (int gpi = 0; gpi < 4; gpi++) {
                    if (!(gpi == 0 || gpi == 3 || gpj == 0 || gpj == 3)) continue;
                    fv[gpi][gpj] = theta * (fv[gpi][gpj] - u0) + u0;
                }
        } else if (active && v == 0 && c >= 0 && c < TXe) {
            flag_error(st, 2u, (long long)map_index(r, D.ny, D.bc) * D.nx + i0 + c);
        }
    }

    if (active) {
#pragma unroll
        for (int gp = 0; gp < 4; gp++) {
            if (c >= 0) S.sxf[c][(4 + gp) * NV + face_slot<NV>(v, c)] = fv[0][gp];     // left face: plus side of face c
            if (c < TX) S.sxf[c + 1][gp * NV + face_slot<NV>(v, c + 1)] = fv[3][gp]; // right face: minus side of face c+1
            if (c >= 0 && c < TX) {
                S.syb[c][gp * NV + face_slot<NV>(v, c)] = fv[gp][0];
                S.syt[r & 1][c][gp * NV + face_slot<NV>(v, c)] = fv[gp][3];
            }
        }
    }
}

// ---- phase 3: Riemann fluxes + Gauss-Lobatto quadrature (src/WENOFV.cpp:1707-1799) -----
// x-faces of row r (when r is an interior row of the item) and y-faces between rows r-1
// and r (when r-1 >= j0-1 and r <= j1).  Four consecutive lanes hold the four Gauss
// points of one face.  FP64_STRICT: lane gp = 0 sums them in the reference's order; the
// contracted build: a reduce-scatter leaves the sum of variable gp on lane gp.
template <int EQ, class R, int FLX, int H, int NT>
__device__ __forceinline__ void phase_riemann(StageSmem<EQ, H, NT> &S, const InstDesc &D, InstState *st, int r, int i0, int j0, int j1,
                                              int TXe)
{
    constexpr int NV = StageGeom<EQ, H, NT>::NV, TX = StageGeom<EQ, H, NT>::TX;
    const int nxf = (r >= j0 && r < j1) ? (TX + 1) * 4 : 0;
    const int nyf = (r >= j0 && r <= j1) ? TX * 4 : 0;
    const int total = nxf + nyf;
    if (total == 0) return;
    const int lane = threadIdx.x & 31, g4 = lane & ~3;
    const double dyr = (r >= j0 && r < j1) ? D.dy[r] : 1.0;
    for (int base = 0; base < total; base += NT) {
        if (base + (int)(threadIdx.x & ~31u) >= total) break; // the whole warp is idle: leave (warp-uniform)
        const int u = base + threadIdx.x;
        const bool act = u < total;
        const int uu = act ? u : total - 1;
        const bool xf = uu < nxf;
        const int f = xf ? (uu >> 2) : ((uu - nxf) >> 2);
        const int gp = uu & 3;
        double UL[NV], UR[NV], F[NV];
        if (xf) {
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const int k = face_slot<NV>(v, f);
                UL[v] = S.sxf[f][gp * NV + k];
                UR[v] = S.sxf[f][(4 + gp) * NV + k];
            }
        } else {
#pragma unroll
            for (int v = 0; v < NV; v++) {
                const int k = face_slot<NV>(v, f);
                UL[v] = S.syt[(r - 1) & 1][f][gp * NV + k];
                UR[v] = S.syb[f][gp * NV + k];
            }
        }
        riemann<EQ, R, FLX>(D.eq, D.flux, UL, UR, F, xf);
        // gWeight = m_gweights_ref[gp] * (cell size) / 2.0 (src/WENOFV.cpp:1774, :1793)
        const double wq = xf ? gl_weight(gp) * dyr / 2.0 : gl_weight(gp) * S.sdxc[f] / 2.0;
        bool bad = false;
#if !WENOFV_STRICT
        if constexpr (NV == 4) {
            // contracted build: a reduce-scatter over the face's 4 lanes, after which lane gp
            // holds the quadrature sum of variable gp, (p0 + p2) + (p1 + p3): three shuffles
            // for the four variables
            double pv[4];
#pragma unroll
            for (int v = 0; v < 4; v++) {
                pv[v] = F[v] * wq;
                bad |= isnan(pv[v]);
            }
            const bool hi = (gp & 2) != 0, odd = (gp & 1) != 0;
            const double k0 = hi ? pv[2] : pv[0], k1 = hi ? pv[3] : pv[1];
            const double s0 = hi ? pv[0] : pv[2], s1 = hi ? pv[1] : pv[3];
            const double r0 = k0 + __shfl_xor_sync(0xffffffffu, s0, 2);
            const double r1 = k1 + __shfl_xor_sync(0xffffffffu, s1, 2);
            const double sum = (odd ? r1 : r0) + __shfl_xor_sync(0xffffffffu, odd ? r0 : r1, 1);
            if (act) {
                if (xf) S.sfx[r & 1][f][gp] = sum;
                else S.sfy[r & 1][f][gp] = sum;
            }
        } else
#endif
        {
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const double pv = F[v] * wq;
            bad |= isnan(pv);
            const double p1 = __shfl_sync(0xffffffffu, pv, g4 + 1);
            const double p2 = __shfl_sync(0xffffffffu, pv, g4 + 2);
            const double p3 = __shfl_sync(0xffffffffu, pv, g4 + 3);
            double ave = 0.0;
            ave += pv;
            ave += p1;
            ave += p2;
            ave += p3;
            if (act && gp == 0) {
                if (xf) S.sfx[r & 1][f][v] = ave;
                else S.sfy[r & 1][f][v] = ave;
            }
        }
        }
        if (bad && act && f < TXe + (xf ? 1 : 0)) flag_error(st, 4u, (long long)map_index(r, D.ny, D.bc) * D.nx + i0 + (f < TXe ? f : TXe - 1));
    }
}

// ---- phase 4: RHS scatter (src/WENOFV.cpp:1802-1827) + SSP-RK combination (:376-473)
//      of row q = r-1, and on the final stage the per-cell CFL step (:486-514) ---------
template <int EQ, int H, int NT>
__device__ __forceinline__ double phase_update(StageSmem<EQ, H, NT> &S, const InstDesc &D, InstState *st, const StageLaunch &L,
                                               int q, int i0, int TXe, double dt, double cmin)
{
    constexpr int NV = StageGeom<EQ, H, NT>::NV, GH = StageGeom<EQ, H, NT>::GH;
    const int t = threadIdx.x;
    const int cu = t / NV, v = t - cu * NV;
    const bool act = cu < TXe;
    const int c = act ? cu : 0;
    const double aL = S.sfx[q & 1][c][v], aR = S.sfx[q & 1][c + 1][v];
    const double aB = S.sfy[q & 1][c][v], aT = S.sfy[(q + 1) & 1][c][v];
    const double dyq = D.dy[q], dxc = S.sdxc[c], dxl = S.sdxl[c];
    double rhs = 0.0;
#if WENOFV_STRICT
    rhs += aL / dxl / dyq;
    rhs += -aR / dxc / dyq;
    rhs += aB / dxc / dyq;
    rhs -= aT / dxc / dyq;
#else
    const double idy = 1.0 / dyq, idxc = S.sidxc[c], idxl = S.sidxl[c];
    rhs = ((aL * idxl - aR * idxc) + (aB - aT) * idxc) * idy;
#endif
    if constexpr (IsTwoPhase<EQ>::value) { // assembleSourceTerm, src/WENOFV.cpp:1831-1872
        if (v == 3 && D.eq.gravity != 0.0) {
            const double rho = S.su[q & 7][0][c + GH] + S.su[q & 7][1][c + GH];
            rhs -= rho * D.eq.gravity;
        }
    }
    const double U = S.su[q & 7][v][c + GH];
    const double Un = L.first_stage ? U : S.sun[q & 1][v][c + GH];
    double Unew;
    if (L.rk1) Unew = U + dt * rhs;
    else Unew = L.A * Un + L.B * U + L.C * dt * rhs;
    const size_t plane = (size_t)D.ny * D.pitch;
    const size_t off = v * plane + (size_t)q * D.pitch + i0 + c;
#if WENOFV_CHECK_BOUNDS
    if (act && (q < 0 || q >= D.ny || i0 + c >= D.nx || off >= (size_t)NV * plane)) {
        flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)q * D.nx + i0 + c);
        return cmin;
    }
#endif
    if (act) {
        if (L.rhs_out) L.rhs_out[off] = rhs;
        else D.buf[L.bout][off] = Unew;
        if (isnan(Unew)) flag_error(st, 8u, (long long)q * D.nx + i0 + c);
    }
    if (L.final_stage && !L.rhs_out) {
        double u[NV];
        const int g = (t & 31) & ~(NV - 1);
#pragma unroll
        for (int k = 0; k < NV; k++) u[k] = __shfl_sync(0xffffffffu, Unew, g + k);
        double ax, ay;
        max_eigs<EQ, double>(D.eq, u, ax, ay);
        const double tmp = D.cfl / (ax / D.dX + ay / D.dY);
        if (act && v == 0) {
            if (isnan(tmp)) flag_error(st, 1u, (long long)q * D.nx + i0 + c);
            else cmin = fmin(cmin, tmp);
        }
    }
    return cmin;
}

// resident CTAs per SM the register allocation is bounded for (measured best).  128 threads:
// the FP64 forms at 3, which keeps all values in registers (4 spills and runs slower), the
// FP32-bulk form at 4 (conservative) or 5 (characteristic, a few spilled values).  256
// threads: 2 (128 registers, a few spilled values), the Euler FP32-bulk form (its flux stays
// FP64) 3
template <int EQ, int RECON, class R, int NT> struct StageMinBlocks {
    static constexpr int value = NT == 256 ? ((sizeof(R) < sizeof(double) && EQ == EQ_EULER) ? 3 : 2)
                                           : (sizeof(R) < sizeof(double) ? (RECON == 1 ? 5 : 4) : 3);
};

// SCH, FLX: the scheme (0 WENO-JS, 1 WENO-Z, 2 WENOEXP) and flux (0 LLF, 1 HLLC) of every
// instance of the launch, as compile-time constants (the engine groups instances by them)
template <int EQ, int RECON, class R, int SCH, int FLX, int NT>
__global__ void __launch_bounds__(NT, StageMinBlocks<EQ, RECON, R, NT>::value) stage_kernel(const StageLaunch L)
{
    static_assert(NT == 128 || (NT == 256 && StageWide<EQ, RECON, R>::value), "stage kernel width");
    constexpr int H = StencilRecon<R, SCH>::H;
    constexpr int TX = StageGeom<EQ, H, NT>::TX;
    using SmemT = StageSmem<EQ, H, NT>;
    static_assert(offsetof(SmemT, sy) % 16 == 0 && offsetof(SmemT, sxf) % 16 == 0, "16-byte exchange loads");
    // the last warp's exchange area (its active cells, from face 8 (NT/32 - 1) on) inside sxf
    static_assert(EqTraits<EQ>::NV != 4 || 8 * (NT / 32 - 1) * SmemT::FS + (TX + 1 - 8 * (NT / 32 - 1)) * 20 + 16 <= (TX + 1) * SmemT::FS,
                  "exchange area of the last warp");
    // the CTA's shared block is dynamic shared memory (it outgrows the 48 KB static limit for
    // wider strips): StageSmem, then StageDynSmem bytes of the primitive ring
    extern __shared__ __align__(16) unsigned char stage_smem_raw[];
    StageSmem<EQ, H, NT> &S = *reinterpret_cast<StageSmem<EQ, H, NT> *>(stage_smem_raw);
    double *stage_dyn_smem = reinterpret_cast<double *>(stage_smem_raw + StageSmemBytes<EQ, H, NT>::value);
    const int nwork = L.counts ? L.counts[0] : L.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = L.work[w];
        const InstDesc &D = L.inst[it.inst];
        InstState *st = &L.state[it.inst];
        if (st->done) continue;
        const double dt = st->dt;
        const int TXe = min(TX, D.nx - it.i0);
#if WENOFV_CHECK_BOUNDS
        if (it.i0 < 0 || it.i0 >= D.nx || it.j0 < 0 || it.j1 > D.ny || it.j0 >= it.j1) { // a malformed work item
            if (threadIdx.x == 0) flag_error(st, 16u /* WENOFV_FLAG_BOUNDS */, (long long)it.j0 * D.nx + it.i0);
            continue;
        }
#endif
        for (int c = threadIdx.x; c < TX; c += NT) {
            const int i = min(it.i0 + c, D.nx - 1);
            S.sdxc[c] = D.dxc[i];
            S.sdxl[c] = D.dxl[i];
#if !WENOFV_STRICT
            S.sidxc[c] = 1.0 / D.dxc[i];
            S.sidxl[c] = 1.0 / D.dxl[i];
#endif
        }
        const double *bin = D.buf[L.bin];
        const double *bun = D.buf[L.bun];
        const bool flag_rows = D.theta_flag != nullptr && L.final_stage && !L.rhs_out;
        // rows j0-1-H .. j0-1+H, the stencils of the first iteration's row
#pragma unroll 1
        for (int m = 0; m <= 2 * H; m++) load_row<EQ, H, NT>(S.su[(it.j0 - 1 - H + m) & 7], bin, D, it.j0 - 1 - H + m, it.i0, st);
        cp_async_commit();
        double cmin = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll 1
        for (int r = it.j0 - 1; r <= it.j1; r++) {
            cp_async_wait_all();
            __syncthreads();
            // row r+H+1 into the slot of row r-H-1 (8 slots: rows r-H .. r+H in use, one in flight)
            if (r + H + 1 <= it.j1 + H) load_row<EQ, H, NT>(S.su[(r + H + 1) & 7], bin, D, r + H + 1, it.i0, st);
            if (!L.first_stage && r >= it.j0 && r < it.j1) load_row<EQ, H, NT>(S.sun[r & 1], bun, D, r, it.i0, st);
            cp_async_commit();
            if (r == it.j0 - 1) { // eigensystems of the first row; later rows come from phase 3
                phase_eigen<EQ, RECON, H, NT>(S, D, r, 0, NT);
                __syncthreads();
            }
            phase_ysweep<EQ, RECON, R, SCH, NT>(S, D, r, stage_dyn_smem, r == it.j0 - 1);
            __syncthreads();
            phase_xsweep<EQ, RECON, R, SCH, NT>(S, D, st, r, it.i0, TXe, stage_dyn_smem, flag_rows && r >= it.j0 && r < it.j1);
            __syncthreads();
            phase_riemann<EQ, R, FLX, H, NT>(S, D, st, r, it.i0, it.j0, it.j1, TXe);
            // the last warp, idle in the second round of Riemann units, prepares the next
            // row's eigensystems (row r+1 is resident; se is not read until the next row)
            if (threadIdx.x >= NT - 32) phase_eigen<EQ, RECON, H, NT>(S, D, r + 1, NT - 32, 32);
            __syncthreads();
            if (r - 1 >= it.j0) cmin = phase_update<EQ, H, NT>(S, D, st, L, r - 1, it.i0, TXe, dt, cmin);
        }
        if (L.final_stage && !L.rhs_out) {
            const double m = block_min(cmin, S.sred);
            if (threadIdx.x == 0) cfl_atomic_min(st, m);
        }
        __syncthreads();
    }
    if (L.final_stage && !L.rhs_out) launch_epilogue(L, FIN_STEP, &S.s_last);
}

// calculateDeltaT of the current state (src/WENOFV.cpp:474-540) for every instance of the
// launch, then the loop bookkeeping (FIN_INIT) by the last CTA.  L.tx: the strip width of the
// launch's work items (that of the instances' stage kernel).
template <int EQ>
__global__ void __launch_bounds__(CFL_NT) cfl_kernel(const StageLaunch L)
{
    constexpr int NV = EqTraits<EQ>::NV, NT = CFL_NT;
    __shared__ double sred[NT / 32];
    __shared__ int s_last;
    const int nwork = L.counts ? L.counts[0] : L.nwork;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = L.work[w];
        const InstDesc &D = L.inst[it.inst];
        InstState *st = &L.state[it.inst];
        if (st->done) continue;
        const double *U = D.buf[st->cur_buf];
        const size_t plane = (size_t)D.ny * D.pitch;
        const int width = min(L.tx, D.nx - it.i0);
        double cmin = __longlong_as_double(0x7ff0000000000000LL);
        for (int e = threadIdx.x; e < width * (it.j1 - it.j0); e += NT) {
            const int j = it.j0 + e / width, i = it.i0 + e % width;
            double u[NV];
#pragma unroll
            for (int k = 0; k < NV; k++) u[k] = U[k * plane + (size_t)j * D.pitch + i];
            double ax, ay;
            max_eigs<EQ, double>(D.eq, u, ax, ay);
            const double tmp = D.cfl / (ax / D.dX + ay / D.dY);
            if (isnan(tmp)) flag_error(st, 1u, (long long)j * D.nx + i);
            else cmin = fmin(cmin, tmp);
        }
        const double m = block_min(cmin, sred);
        if (threadIdx.x == 0) cfl_atomic_min(st, m);
        __syncthreads();
    }
    launch_epilogue(L, FIN_INIT, &s_last);
}

} // namespace strict / fast
} // namespace wenofv
