// solver3d.cu — host orchestration of the 3D forging increment on the GPU and its C ABI (ifea3d_*).
//
// The control flow is Forging3DSolver's (ThreeD/Forging3DSolver.cs:540-1537): the host runs the increment
// loop, the Newton iteration, the line search and the PCG loop, and reads back only the handful of scalars
// those decisions need; every array operation is a device kernel on the context's stream.
#include <chrono>
#include <climits>
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <future>
#include <thread>
#include <vector>

#include "common.cuh"
#include "remesh.h"
#include "trimesh.h"
#include "warmstart.h"
#include "kernels3d.cuh"
#include "mesh3d.h"
#include "runtime.cuh"
#include "multifrontal.cuh"

namespace ifea {

static std::string fmt(const char *f, ...) __attribute__((format(printf, 1, 2)));
static std::string fmt(const char *f, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

// Adds the wall time of a scope to an accumulator (the phases end in a stream synchronisation, so host time
// is the phase's time); the split mirrors Forging3DSolver.TimingSummary (:1924-1943).
// ------------------------------------------------------------------ learned warm start (inputs, targets, guess)
// The network replaces LoadVelocityGuess (Forging3DSolver.cs:854-869): from each node's state at the start of
// an increment it predicts the change of the node's global velocity over the increment. Its 16 inputs per node
// (FP32): the previous converged velocity and its change over the increment before (both / ram); the node's
// mean effective strain and mean strain rate (/ the reference rate) over its tets; the contact state as one-hot
// (free, bottom die, top die); the clearances to both dies (/ h, clamped to [-1, 4]); the stroke increment (/ h);
// the radial and axial position (/ the billet size). v0 keeps the velocity the prediction is added to.
__global__ void k_ws_features(View3 V, float *__restrict__ F, double *__restrict__ v0, double rate_ref, double h,
                              double ds, double size, int have_prev)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 g = ld3(V.vg, n), gp = have_prev ? ld3(V.vg_prev, n) : g;
        st3(v0, n, g);
        double e = 0, r = 0;
        int cnt = V.nts[n + 1] - V.nts[n];
        for (int32_t q = V.nts[n]; q < V.nts[n + 1]; q++) {
            int t = V.ntl[q];
            e += V.eps[t];
            r += V.el_rate[t];
        }
        if (cnt) {
            e /= cnt;
            r /= cnt;
        }
        d3 p = ld3(V.x, n);
        double cb = hf_clearance(V.die[0], p, 0), ct = hf_clearance(V.die[1], p, V.gap);
        int c = V.contact[n];
        float *f = F + 16 * (int64_t)n;
        f[0] = (float)(g.x / V.ram); f[1] = (float)(g.y / V.ram); f[2] = (float)(g.z / V.ram);
        f[3] = (float)((g.x - gp.x) / V.ram); f[4] = (float)((g.y - gp.y) / V.ram); f[5] = (float)((g.z - gp.z) / V.ram);
        f[6] = (float)e;
        f[7] = (float)(r / rate_ref);
        f[8] = c == IFEA_FREE; f[9] = c == IFEA_BOTTOM_DIE; f[10] = c == IFEA_TOP_DIE;
        f[11] = (float)rclamp(cb / h, -1.0, 4.0);
        f[12] = (float)rclamp(ct / h, -1.0, 4.0);
        f[13] = (float)(ds / h);
        f[14] = (float)(sqrt(p.x * p.x + p.y * p.y) / size);
        f[15] = (float)(p.z / size);
    }
}

// training target of an accepted increment: the change of the global velocity over it, / ram
__global__ void k_ws_targets(View3 V, const double *__restrict__ v0, float *__restrict__ T)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 g = ld3(V.vg, n), a = ld3(v0, n);
        T[3 * (int64_t)n] = (float)((g.x - a.x) / V.ram);
        T[3 * (int64_t)n + 1] = (float)((g.y - a.y) / V.ram);
        T[3 * (int64_t)n + 2] = (float)((g.z - a.z) / V.ram);
    }
}

// the predicted start: v0 + ram * prediction, in the nodal frames, fixed DOFs overwritten (as k_guess)
__global__ void k_ws_guess(View3 V, const double *__restrict__ v0, const float *__restrict__ Y, double *__restrict__ out)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 a = ld3(v0, n);
        d3 g = mk3(a.x + V.ram * (double)Y[3 * (int64_t)n], a.y + V.ram * (double)Y[3 * (int64_t)n + 1],
                   a.z + V.ram * (double)Y[3 * (int64_t)n + 2]);
        d3 l = to_local(V, n, g);
        for (int c = 0; c < 3; c++) {
            int d = 3 * n + c;
            out[d] = V.fixed[d] ? V.fixed_val[d] : get3(l, c);
        }
    }
}

// One pass of low-pass filtering of the predicted velocity change over the mesh: each node takes the mean, over its
// tets, of the tets' nodal means. The network predicts every node on its own; its pointwise noise is not
// divergence-free and the penalty term of the functional punishes exactly that, so the prediction is smoothed
// before it is weighed against the reference start.
__global__ void k_ws_smooth(View3 V, const float *__restrict__ Y, float *__restrict__ out)
{
    GRID_STRIDE(n, V.nn)
    {
        float acc[3] = {0, 0, 0};
        int cnt = V.nts[n + 1] - V.nts[n];
        for (int32_t q = V.nts[n]; q < V.nts[n + 1]; q++) {
            const int32_t *t = V.tets + 4 * (int64_t)V.ntl[q];
            for (int a = 0; a < 4; a++)
                for (int c = 0; c < 3; c++) acc[c] += 0.25f * Y[3 * (int64_t)t[a] + c];
        }
        for (int c = 0; c < 3; c++) out[3 * (int64_t)n + c] = cnt ? acc[c] / cnt : Y[3 * (int64_t)n + c];
    }
}

// out = a + s (b - a), elementwise
__global__ void k_ws_mix(int n, const double *__restrict__ a, const double *__restrict__ b, double s, double *__restrict__ out)
{
    GRID_STRIDE(i, n) { out[i] = a[i] + s * (b[i] - a[i]); }
}

// ------------------------------------------------------------------ FillPercent (:2149-2189) on the device
// The reference builds a TetLocator over the current mesh every step (a bucket grid of cell 2 h over the nodes'
// bounding box, every tet listed in each cell its bounding box touches) and counts the closed cavity's sample points
// that lie in some tet (barycentric weights all >= -1e-9 in a tet of positive volume). Here the grid is built by
// counting, a one-block prefix sum and a fill, and one thread tests each sample point against its cell's tets.
struct LocGrid {
    double x0, y0, z0, cell;
    int nx, ny, nz;
};

__global__ void k_node_box(View3 V)
{
    double mx[6] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY, -INFINITY, -INFINITY};
    GRID_STRIDE(n, V.nn)
    {
        d3 p = ld3(V.x, n);
        mx[0] = rmax(mx[0], p.x); mx[1] = rmax(mx[1], p.y); mx[2] = rmax(mx[2], p.z);
        mx[3] = rmax(mx[3], -p.x); mx[4] = rmax(mx[4], -p.y); mx[5] = rmax(mx[5], -p.z);
    }
    const int s6[6] = {S_BOX0, S_BOX1, S_BOX2, S_BOX3, S_BOX4, S_BOX5};
    emit_max<6>(V, mx, s6);
}

__device__ __forceinline__ int loc_axis(double v, double v0, double cell, int n)
{
    return iclamp((int)((v - v0) / cell), 0, n - 1);
}

// mode 0: count the tets of every cell (into count[c + 1]); mode 1: list them (slot from fill[c])
__global__ void k_loc_tets(View3 V, LocGrid G, int mode, int32_t *__restrict__ count, int32_t *__restrict__ fill,
                           int32_t *__restrict__ items)
{
    GRID_STRIDE(e, V.ne)
    {
        const int32_t *t = V.tets + 4 * e;
        d3 lo = ld3(V.x, t[0]), hi = lo;
        for (int a = 1; a < 4; a++) {
            d3 p = ld3(V.x, t[a]);
            lo = mk3(rmin(lo.x, p.x), rmin(lo.y, p.y), rmin(lo.z, p.z));
            hi = mk3(rmax(hi.x, p.x), rmax(hi.y, p.y), rmax(hi.z, p.z));
        }
        int i0 = loc_axis(lo.x, G.x0, G.cell, G.nx), i1 = loc_axis(hi.x, G.x0, G.cell, G.nx);
        int j0 = loc_axis(lo.y, G.y0, G.cell, G.ny), j1 = loc_axis(hi.y, G.y0, G.cell, G.ny);
        int k0 = loc_axis(lo.z, G.z0, G.cell, G.nz), k1 = loc_axis(hi.z, G.z0, G.cell, G.nz);
        for (int k = k0; k <= k1; k++)
            for (int j = j0; j <= j1; j++)
                for (int i = i0; i <= i1; i++) {
                    int c = (k * G.ny + j) * G.nx + i;
                    if (mode == 0) atomicAdd(count + c + 1, 1);
                    else items[atomicAdd(fill + c, 1)] = e;
                }
    }
}

// inclusive prefix sum of a[0..n) in one block (n is a few thousand cells), fill = a copy of it
__global__ void k_scan_block(int32_t *__restrict__ a, int n, int32_t *__restrict__ fill)
{
    __shared__ int32_t carry;
    __shared__ int32_t part[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        int i = base + threadIdx.x;
        part[threadIdx.x] = i < n ? a[i] : 0;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int32_t v = threadIdx.x >= off ? part[threadIdx.x - off] : 0;
            __syncthreads();
            part[threadIdx.x] += v;
            __syncthreads();
        }
        if (i < n) {
            a[i] = part[threadIdx.x] + carry;
            fill[i] = a[i];
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry += part[1023];
        __syncthreads();
    }
}

__global__ void k_fill_query(View3 V, LocGrid G, const int32_t *__restrict__ start, const int32_t *__restrict__ items,
                             const double *__restrict__ pts, int np)
{
    double acc[1] = {0};
    GRID_STRIDE(q, np)
    {
        d3 p = ld3(pts, q);
        int c = (loc_axis(p.z, G.z0, G.cell, G.nz) * G.ny + loc_axis(p.y, G.y0, G.cell, G.ny)) * G.nx +
                loc_axis(p.x, G.x0, G.cell, G.nx);
        for (int32_t k = start[c]; k < start[c + 1]; k++) {
            const int32_t *t = V.tets + 4 * items[k];
            d3 a = ld3(V.x, t[0]), b = ld3(V.x, t[1]), cc = ld3(V.x, t[2]), d = ld3(V.x, t[3]);
            double v = tet_volume(a, b, cc, d);
            if (v <= 0) continue;
            double b0 = tet_volume(p, b, cc, d) / v, b1 = tet_volume(a, p, cc, d) / v, b2 = tet_volume(a, b, p, d) / v;
            double b3 = 1 - b0 - b1 - b2;
            if (b0 >= -1e-9 && b1 >= -1e-9 && b2 >= -1e-9 && b3 >= -1e-9) {
                acc[0] += 1;
                break;
            }
        }
    }
    const int s1[1] = {S_FILL};
    emit_sum<1>(V, acc, s1);
}

struct PhaseTimer {
    double &acc;
    std::chrono::steady_clock::time_point t0;
    explicit PhaseTimer(double &a) : acc(a), t0(std::chrono::steady_clock::now()) {}
    ~PhaseTimer() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

__global__ void k_die_query(HField d, int n, const double *p, double offset, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        d3 q = ld3(p, i), nrm;
        double *o = out + 8 * (size_t)i;
        o[0] = hf_clearance(d, q, offset);
        d3 r = hf_project(d, q, offset, &nrm);
        o[1] = r.x, o[2] = r.y, o[3] = r.z, o[4] = nrm.x, o[5] = nrm.y, o[6] = nrm.z;
        o[7] = hf_height(d, q.x, q.y);
    }
}

struct Forging3D {
    ifea3d_params P;
    double t_trigger = 0, t_prepare = 0, t_assemble = 0, t_linesearch = 0, t_factor = 0, t_pcg = 0, t_final = 0,
           t_update = 0, t_total = 0;
    cudaStream_t st = nullptr;
    std::string err;
    // constants (Forging3DSolver.cs:137-150)
    double rate_ref = 0, rate_cut = 0, sig_ref = 0, k_pen = 0, u0 = 0, h = 0;
    // increment state
    double gap0 = 0, gap = 0, ds_cur = 0, time = 0, last_rel = INFINITY, vol0 = 0;
    int step_index = 0, warm = 0, recovery_pass = 0;
    bool have_vg_prev = false, initialized = false;
    int iterations = 0, n_fact = 0, n_pcg = 0, remesh_requests = 0, projection_reverts = 0, corner_penetrations = 0;
    int last_cutbacks = 0, n_newton = 0, n_assemble = 0, lin_its = 0;
    double load = 0, reaction = 0, power = 0, last_dt = 0, rnorm = 0, beta_last = 0, max_diag = 0;
    // linear solver (SolveLinear :965-1019)
    std::unique_ptr<LinearSolver> lin;
    // Symbolic analysis of the pattern, started on a host thread when the mesh is set and taken by the first
    // factorisation; the job reads only topo's pattern and node_xyz, which nothing writes meanwhile. Node order
    // (`ordering`): 1 (default) the library's coordinate nested dissection with minimum-vertex-cover separators
    // at the top levels (21 ms instead of METIS's 86 ms on the 31.9k-tet case, and a shorter panel chain:
    // 105 steps against 115); 0 METIS through cuSOLVER.
    std::thread sym_job;
    std::unique_ptr<MfSymbolic> sym_pre;
    std::string sym_err;
    // a remesh starts the job as soon as the new connectivity is known: it builds that mesh's topology first
    // (handed to set_mesh through topo_ready) and then analyses its pattern
    std::unique_ptr<TetTopology> topo_ahead;
    std::vector<double> ahead_x;
    std::vector<int32_t> ahead_t;
    std::vector<uint8_t> ahead_onx, ahead_ony;
    std::promise<std::string> topo_promise;
    std::future<std::string> topo_ready;
    bool ahead_pending = false;
    double t_sym_wait = 0;
    int ordering = 1;
    std::vector<double> node_xyz;  // node coordinates when the mesh was set
    bool need_analyze = true, have_factor = false;
    // single-precision factor refined by FP64 PCG (off: the reference's FP64 direct solve after a factorisation)
    bool factor_fp32 = false;
    int fp32_fallbacks = 0, refine_its = 0;
    // give up a reused-factor PCG as soon as its contraction rate shows it cannot meet the budget, and try a factor
    // from an earlier increment again only now and then once that failed (on with the single-precision factor;
    // off in the reference's FP64 form, whose iteration counts it must reproduce)
    bool pcg_early_abort = false;
    double pcg_budget_scale = 2.0;  // factorisations' worth of PCG iterations a reused factor may take
    // Inexact Newton (off by default; the reference solves every linear system to 1e-7): with pcg_forcing f > 0 a
    // Newton iteration's PCG stops at the relative residual f x the previous iteration's update norm, clamped to
    // [1e-7, 1e-3] (1e-3 for the first iteration of an increment)
    double pcg_forcing = 0;
    double lin_tol = 1e-7;  // the PCG tolerance of the linear solve in progress
    int factor_step = -1, stale_failures = 0;  // increment of the cached factor; failed tries of a stale one
    int wide_rows = mf::kWideM;  // fronts at least this tall use the multi-CTA solve path
    // learned warm start: mode bit 1 records (inputs, target) of every accepted increment into the network's
    // training set, bit 2 starts each increment from the network's prediction when its energy is lower than
    // the reference start's (else the reference start is kept)
    // remeshing (RemeshCore, Forging3DSolver.cs:1958-2101) on the host where the reference remeshes; off by
    // default, so that increments stay comparable with the oracle, which counts the requests instead
    bool remesh_enabled = false;
    int remesh_count = 0, remesh_rejected = 0, refinement_levels = 1, max_nodes = 1 << 30;
    double t_remesh = 0;
    double t_rm_stuff = 0, t_rm_refine = 0, t_rm_place = 0, t_rm_remap = 0, t_rm_setmesh = 0;  // remesh phases
    std::vector<HotSpot> hot;        // places where increments failed (later remeshes refine there)
    d3 fail_at = mk3(0, 0, 0);
    bool have_fail_at = false;
    std::vector<double> die_host[2];  // host copies of the die heights (the remesher's clearances)
    TriMeshHost tm_host[2];            // triangulated dies: host grids (the remesher's), device copies below
    DBuf<double> tm_v[2];
    DBuf<int32_t> tm_t[2], tm_xys[2], tm_xyi[2], tm_g3s[2], tm_g3i[2];
    std::string last_remesh;
    DBuf<double> d_cavity;          // the closed cavity's sample points (FillPercent)
    DBuf<int32_t> d_loc_start, d_loc_fill, d_loc_items;
    WarmStartNet *ws_net = nullptr;
    int ws_mode = 0, ws_used = 0, ws_fallbacks = 0;
    // 0: the lower-functional start of the two; 1: the network's start always; 2: a step along the prediction
    // from the reference start, chosen on the functional (the reference start when no step lowers it)
    int ws_policy = 0;
    int ws_smooth = 2;  // smoothing passes over the prediction (k_ws_smooth)
    double ws_last_step = 0;
    DBuf<float> d_wsf, d_wst, d_wsy, d_wsy2;
    DBuf<double> d_wsv0, d_wstry;
    int pcg_failures = 0, pcg_skip = 0, pcg_failures_total = 0;
    // mesh
    TetTopology topo;
    int have_dies = 0;
    HField die[2];
    DBuf<double> die_h[2];
    // device arrays
    DBuf<int32_t> d_tets, d_nts, d_ntl, d_qk, d_gslot, d_bface, d_bowner, d_nfs, d_nfl, d_nbr_start, d_nbr, d_diag,
        d_gstart, d_gnode, d_kvs, d_kvn, d_kvpj, d_kvks, d_kvk, d_nfix, d_dieaxis, d_err, d_counters;
    DBuf<int8_t> d_ntl_local;
    DBuf<uint8_t> d_bsym, d_surf, d_onx, d_ony, d_fixed, d_contact, d_release, d_cT, d_bad;
    DBuf<double> d_hloc, d_x, d_xT, d_vg, d_vgprev, d_ax, d_fixedval, d_kfric, d_afric, d_grad, d_vol, d_vnode,
        d_gcoef, d_clocal, d_kvol, d_val, d_eps, d_dmg, d_elsig, d_elrate, d_eldev, d_elmean, d_vbuf[2], d_r, d_b,
        d_dv, d_er, d_eg, d_ew, d_eenergy, d_epower, d_partials, d_scalars, d_nrm, d_pred, d_nodal, d_q, d_pr, d_pz,
        d_pp, d_pq;
    int vcur = 0;
    HostPinned<double> hs;
    HostPinned<int32_t> hi;
    int wpb = 8;          // warps per block of the column kernels
    size_t col_smem = 0;  // dynamic shared memory of the column kernels

    Forging3D(const ifea3d_params &p) : P(p)
    {
        cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        h = P.h;
        ds_cur = P.ds;
        rate_ref = P.ram / P.size;
        rate_cut = 1e-3 * rate_ref;
        sig_ref = flow_stress(P.C, P.N, P.M, P.eps0, 0, rate_ref);
        k_pen = P.penalty_factor * sig_ref / rate_ref;
        u0 = 5e-3 * P.ram;
        hs.resize(S_COUNT + 8);
        hi.resize(8);
        d_partials.resize((size_t)S_COUNT * kReduceBlocks);
        d_scalars.resize(S_COUNT);
        d_err.resize(4);
        d_counters.resize(4);
        lin.reset(new MfSolver(st));
    }
    bool own_stream = true;
    ~Forging3D()
    {
        join_analysis();
        if (st) cudaStreamSynchronize(st);
        lin.reset();
        if (st && own_stream) cudaStreamDestroy(st);
    }

    // Run on a caller-provided stream from now on (the context's own stream is kept for destruction order).
    void set_stream(cudaStream_t s)
    {
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (own_stream) cudaStreamDestroy(st);
        own_stream = false;
        st = s;
        lin->set_stream(s);
    }

    int grid(int n) const { return std::max(1, std::min((n + 255) / 256, 8 * 148)); }

    // Switch the factorisation between double and single precision; the next solve analyses and factorises anew.
    void use_precision(bool fp32)
    {
        if (fp32 == (lin->value_bytes() == 4)) return;
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        lin.reset();
        if (fp32)
            lin.reset(new MfSolverT<float>(st));
        else
            lin.reset(new MfSolverT<double>(st));
        lin->set_wide_rows(wide_rows);
        need_analyze = true;
        have_factor = false;
        pcg_skip = pcg_failures = 0;
    }

    View3 view()
    {
        View3 V;
        memset(&V, 0, sizeof V);
        V.nn = topo.nn; V.ne = topo.ne; V.ndof = topo.ndof; V.nbf = (int)topo.bowner.size();
        V.tets = d_tets; V.nts = d_nts; V.ntl = d_ntl; V.qk = d_qk; V.gslot = d_gslot; V.bface = d_bface;
        V.bowner = d_bowner; V.nfs = d_nfs; V.nfl = d_nfl; V.ntl_local = d_ntl_local; V.bsym = d_bsym;
        V.is_surface = d_surf; V.on_x0 = d_onx; V.on_y0 = d_ony; V.nbr_start = d_nbr_start; V.nbr = d_nbr;
        V.diag_slot = d_diag; V.g_start = d_gstart; V.g_node = d_gnode; V.kv_start = d_kvs; V.kv_n = d_kvn;
        V.kv_pj = d_kvpj; V.kv_kstart = d_kvks; V.kv_k = d_kvk; V.h_local = d_hloc;
        V.x = d_x; V.vg = d_vg; V.vg_prev = d_vgprev; V.ax = d_ax; V.fixed_val = d_fixedval; V.k_fric = d_kfric;
        V.a_fric = d_afric; V.grad = d_grad; V.vol = d_vol; V.v_node = d_vnode; V.g_coef = d_gcoef; V.c_local = d_clocal;
        V.kvol = d_kvol; V.val = d_val; V.eps = d_eps; V.dmg = d_dmg; V.el_sig = d_elsig; V.el_rate = d_elrate;
        V.el_dev = d_eldev; V.el_mean = d_elmean; V.v = d_vbuf[vcur]; V.v_trial = d_vbuf[1 - vcur]; V.r = d_r; V.b = d_b;
        V.dv = d_dv; V.e_r = d_er; V.e_g = d_eg; V.e_w = d_ew; V.e_energy = d_eenergy; V.e_power = d_epower;
        V.n_fix = d_nfix; V.die_axis = d_dieaxis; V.fixed = d_fixed; V.contact = d_contact; V.release = d_release;
        V.partials = d_partials; V.scalars = d_scalars; V.err = d_err;
        V.die[0] = die[0]; V.die[1] = die[1];
        V.C = P.C; V.N = P.N; V.M = P.M; V.eps0 = P.eps0; V.friction = P.friction; V.ram = P.ram;
        V.rate_cut = rate_cut; V.k_pen = k_pen; V.u0 = u0; V.newton_blend = P.newton_blend; V.gap = gap;
        return V;
    }

    // ---------------------------------------------------------------- reductions / readback
    void finalize(std::initializer_list<int> codes)
    {
        SlotList l;
        l.n = 0;
        for (int c : codes) l.code[l.n++] = c;
        k_finalize<<<l.n, 256, 0, st>>>(d_partials, d_scalars, l);
    }
    static int MAXS(int slot) { return slot | (1 << 16); }
    const double *read_scalars()
    {
        cuda_check(cudaMemcpyAsync(hs.p, d_scalars.p, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H scalars");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        return hs.p;
    }
    void reset_err()
    {
        int32_t v[4] = {INT_MAX, INT_MAX, 0, 0};
        cuda_check(cudaMemcpyAsync(d_err.p, v, sizeof v, cudaMemcpyHostToDevice, st), "H2D err");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }
    void read_err(int32_t *out4)
    {
        cuda_check(cudaMemcpyAsync(hi.p, d_err.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "D2H err");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        memcpy(out4, hi.p, 4 * sizeof(int32_t));
    }

    // ---------------------------------------------------------------- setup
    void join_analysis()
    {
        if (sym_job.joinable()) sym_job.join();
    }

    // one analysis of tp's pattern on the calling (job) thread: coordinate order when xyz is given, else METIS
    void analysis_job(int dev, const TetTopology *tp, const double *xyz, std::unique_ptr<MfSymbolic> *out,
                      std::string *err)
    {
        const int ndof = tp->ndof;
        const int32_t *cp = tp->col_ptr.data(), *ri = tp->row_idx.data();
        analysis_job(dev, ndof, cp, ri, xyz, out, err, tp->nbr_start.data(), tp->nbr.data());
    }
    // the pattern (cp, ri) is the topology's full 3 x 3 block pattern of the node lists (node_start, node_list)
    void analysis_job(int dev, int ndof, const int32_t *cp, const int32_t *ri, const double *xyz,
                      std::unique_ptr<MfSymbolic> *out, std::string *err, const int32_t *node_start,
                      const int32_t *node_list)
    {
        cusolverSpHandle_t hsp = nullptr;
        cusparseMatDescr_t descr = nullptr;
        try {
            cudaSetDevice(dev);
            if (!xyz && cusolverSpCreate(&hsp) != CUSOLVER_STATUS_SUCCESS) {
                hsp = nullptr;
                *err = "cusolverSpCreate failed";
            } else if (cusparseCreateMatDescr(&descr) != CUSPARSE_STATUS_SUCCESS) {
                descr = nullptr;
                *err = "cusparseCreateMatDescr failed";
            } else {
                cusparseSetMatType(descr, CUSPARSE_MATRIX_TYPE_GENERAL);
                cusparseSetMatIndexBase(descr, CUSPARSE_INDEX_BASE_ZERO);
                std::unique_ptr<MfSymbolic> S(new MfSymbolic);
                std::string e = S->analyze(ndof, cp, ri, 3, hsp, descr, xyz, node_start, node_list);
                if (e.empty())
                    *out = std::move(S);
                else
                    *err = e;
            }
        } catch (std::exception &x) {
            *err = x.what();
        } catch (...) {
            *err = "symbolic analysis failed";
        }
        if (descr) cusparseDestroyMatDescr(descr);
        if (hsp) cusolverSpDestroy(hsp);
    }

    void start_analysis()
    {
        join_analysis();
        sym_pre.reset();
        sym_err.clear();
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        const double *xyz = ordering == 1 ? node_xyz.data() : nullptr;
        sym_job = std::thread([this, dev, xyz] { analysis_job(dev, &topo, xyz, &sym_pre, &sym_err); });
    }

    // The remesher's topology hook: the new mesh's topology and symbolic analysis on the job thread, while the
    // remesher places and remaps. The analysis orders by the nodes' stuffed positions (the order only shapes the
    // fill); set_mesh takes the topology when it is handed the same tets.
    void start_ahead(const std::vector<d3> &x, const std::vector<int32_t> &t, const std::vector<uint8_t> &onx,
                     const std::vector<uint8_t> &ony)
    {
        join_analysis();
        sym_pre.reset();
        sym_err.clear();
        int dev = 0;
        cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
        ahead_x.resize(3 * x.size());
        for (size_t n = 0; n < x.size(); n++) st3(ahead_x.data(), (int)n, x[n]);
        ahead_t = t;
        ahead_onx = onx;
        ahead_ony = ony;
        // the topology replaced at the last remesh is rebuilt in place: its buffers (the 3 x 3 block pattern is a few
        // hundred MB on a 200k-tet mesh) are reused instead of being allocated and faulted in again
        if (!topo_ahead) topo_ahead.reset(new TetTopology);
        topo_promise = std::promise<std::string>();
        topo_ready = topo_promise.get_future();
        ahead_pending = true;
        const bool xyz = ordering == 1;
        sym_job = std::thread([this, dev, xyz] {
            std::string e;
            try {
                e = topo_ahead->build((int)(ahead_x.size() / 3), (int)(ahead_t.size() / 4), ahead_x.data(),
                                      ahead_t.data(), ahead_onx.data(), ahead_ony.data());
            } catch (std::exception &x) {
                e = x.what();
            }
            // the pattern's addresses are taken before set_mesh may swap the topology in (the buffers move with it)
            const int ndof = topo_ahead->ndof;
            const int32_t *cp = topo_ahead->col_ptr.data(), *ri = topo_ahead->row_idx.data();
            const int32_t *ns = topo_ahead->nbr_start.data(), *nl = topo_ahead->nbr.data();
            topo_promise.set_value(e);
            if (!e.empty()) {
                sym_err = e;
                return;
            }
            analysis_job(dev, ndof, cp, ri, xyz ? ahead_x.data() : nullptr, &sym_pre, &sym_err, ns, nl);
        });
    }

    // the analysis for the next factorisation: the one started with the mesh when it is there, else made now
    void analyze_pattern()
    {
        if (sym_job.joinable() || sym_pre || !sym_err.empty()) {
            {
                PhaseTimer pt(t_sym_wait);
                join_analysis();
            }
            if (!sym_pre) {
                std::string e = sym_err.empty() ? "symbolic analysis failed" : sym_err;
                sym_err.clear();
                throw Failure(IFEA_INPUT_INVALID, e);
            }
            lin->analyze_from(std::move(*sym_pre));
            sym_pre.reset();
        } else {
            lin->analyze(topo.ndof, topo.col_ptr.data(), topo.row_idx.data(), 3, ordering == 1 ? node_xyz.data() : nullptr);
        }
    }

    void set_mesh(int nn, int ne, const double *x, const int32_t *tets, const uint8_t *ox, const uint8_t *oy)
    {
        // the topology built ahead for these tets (a remesh), its analysis still running; else both made here
        bool ahead = ahead_pending && ahead_t.size() == 4 * (size_t)ne && ahead_x.size() == 3 * (size_t)nn &&
                     std::equal(ahead_t.begin(), ahead_t.end(), tets) &&
                     std::equal(ahead_onx.begin(), ahead_onx.end(), ox) && std::equal(ahead_ony.begin(), ahead_ony.end(), oy);
        if (ahead) {
            ahead_pending = false;
            std::string e = topo_ready.get();
            if (!e.empty()) {
                join_analysis();
                throw Failure(IFEA_INPUT_INVALID, e);
            }
            std::swap(topo, *topo_ahead);
            node_xyz.assign(x, x + 3 * (size_t)nn);
        } else {
            join_analysis();
            ahead_pending = false;
            sym_pre.reset();
            sym_err.clear();
            std::string e = topo.build(nn, ne, x, tets, ox, oy);
            if (!e.empty()) throw Failure(IFEA_INPUT_INVALID, e);
            node_xyz.assign(x, x + 3 * (size_t)nn);
            start_analysis();
        }
        std::vector<double> hl = local_lengths(topo, x, h);
        d_tets.upload(topo.tets, st); d_nts.upload(topo.nts, st); d_ntl.upload(topo.ntl, st); d_qk.upload(topo.qk, st);
        d_gslot.upload(topo.gslot, st); d_bface.upload(topo.bface, st); d_bowner.upload(topo.bowner, st);
        d_nfs.upload(topo.nfs, st); d_nfl.upload(topo.nfl, st); d_ntl_local.upload(topo.ntl_local, st);
        d_bsym.upload(topo.bsym, st); d_surf.upload(topo.is_surface, st); d_onx.upload(topo.on_x0, st);
        d_ony.upload(topo.on_y0, st); d_nbr_start.upload(topo.nbr_start, st); d_nbr.upload(topo.nbr, st);
        d_diag.upload(topo.diag_slot, st); d_gstart.upload(topo.g_start, st); d_gnode.upload(topo.g_node, st);
        d_kvs.upload(topo.kv_start, st); d_kvn.upload(topo.kv_n, st); d_kvpj.upload(topo.kv_pj, st);
        d_kvks.upload(topo.kv_kstart, st); d_kvk.upload(topo.kv_k, st); d_hloc.upload(hl, st);
        d_x.upload(x, 3 * (size_t)nn, st);
        size_t N3 = 3 * (size_t)nn, ndof = topo.ndof, G = topo.g_node.size();
        d_xT.resize(N3); d_vg.resize(N3); d_vgprev.resize(N3); d_ax.resize(9 * (size_t)nn); d_fixedval.resize(ndof);
        d_kfric.resize(nn); d_afric.resize(nn); d_grad.resize(12 * (size_t)ne); d_vol.resize(ne); d_vnode.resize(nn);
        d_gcoef.resize(3 * G); d_clocal.resize(3 * G); d_kvol.resize(topo.nnz); d_val.resize(topo.nnz);
        d_eps.resize(ne); d_dmg.resize(ne); d_elsig.resize(ne); d_elrate.resize(ne); d_eldev.resize(6 * (size_t)ne);
        d_elmean.resize(ne); d_vbuf[0].resize(ndof); d_vbuf[1].resize(ndof); d_r.resize(ndof); d_b.resize(ndof);
        d_dv.resize(ndof); d_er.resize(12 * (size_t)ne); d_eg.resize(12 * (size_t)ne); d_ew.resize(2 * (size_t)ne);
        d_eenergy.resize(ne); d_epower.resize(ne); d_nrm.resize(N3); d_pred.resize(N3); d_nodal.resize(nn);
        d_q.resize(ne); d_pr.resize(ndof); d_pz.resize(ndof); d_pp.resize(ndof); d_pq.resize(ndof);
        d_nfix.resize(nn); d_dieaxis.resize(nn); d_fixed.resize(ndof); d_contact.resize(nn); d_release.resize(nn);
        d_cT.resize(nn); d_bad.resize(nn);
        for (auto *b : {&d_vg, &d_vgprev, &d_eps, &d_dmg, &d_elmean, &d_eldev, &d_vbuf[0], &d_vbuf[1], &d_r, &d_b, &d_dv})
            b->zero(st);
        d_contact.zero(st); d_release.zero(st); d_fixed.zero(st); d_fixedval.zero(st); d_nfix.zero(st);
        d_dieaxis.zero(st); d_kvol.zero(st); d_val.zero(st);
        std::vector<double> sig(ne, sig_ref);
        d_elsig.upload(sig, st);
        d_elrate.zero(st);
        // column-kernel launch shape: chunk of 9*max_nbr doubles per warp in shared memory
        size_t per_warp = 9 * (size_t)topo.max_nbr * sizeof(double);
        wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (160 * 1024) / std::max<size_t>(per_warp, 1)));
        col_smem = per_warp * wpb;
        if (per_warp > 200 * 1024) throw Failure(IFEA_INPUT_INVALID, "node neighbourhood too large for the column kernel");
        auto set_smem = [&](const void *f) {
            ensure_dynamic_smem(f, (int)col_smem);
        };
        set_smem((const void *)k_columns<ASM_MATRIX, true>);
        set_smem((const void *)k_columns<ASM_MATRIX, false>);
        set_smem((const void *)k_columns<ASM_RESIDUAL, false>);
        set_smem((const void *)k_columns<ASM_ENERGY, false>);
        set_smem((const void *)k_kvol);
        need_analyze = true;
        have_factor = false;
        pcg_failures = pcg_skip = 0;
        vcur = 0;
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }

    // a die given as a closed triangulated solid (TriMeshDie, ThreeD/TriMeshSolid.cs:248-297), in its closed
    // position for the top die like the height field
    void set_trimesh_die(int side, int nv, const double *v, int nt, const int32_t *tri)
    {
        if (side < 0 || side > 1) throw Failure(IFEA_INPUT_INVALID, "invalid die side");
        TriMeshHost &h = tm_host[side];
        std::string e = h.build(nv, v, nt, tri);
        if (!e.empty()) throw Failure(IFEA_INPUT_INVALID, e);
        tm_v[side].upload(h.v, st); tm_t[side].upload(h.t, st);
        tm_xys[side].upload(h.xy_start, st); tm_xyi[side].upload(h.xy_items.empty() ? std::vector<int32_t>{0} : h.xy_items, st);
        tm_g3s[side].upload(h.g3_start, st); tm_g3i[side].upload(h.g3_items.empty() ? std::vector<int32_t>{0} : h.g3_items, st);
        HField &d = die[side];
        d.side = side;
        d.kind = 1;
        d.nx = d.ny = 1;
        d.x0 = h.grid.mn[0]; d.y0 = h.grid.mn[1]; d.dx = h.grid.c2;
        d.h = nullptr;
        d.tm = h.grid;
        d.tm.v = tm_v[side].p; d.tm.t = tm_t[side].p;
        d.tm.xy_start = tm_xys[side].p; d.tm.xy_items = tm_xyi[side].p;
        d.tm.g3_start = tm_g3s[side].p; d.tm.g3_items = tm_g3i[side].p;
        die_host[side].clear();
        have_dies |= 1 << side;
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }

    // Clearance, Project and SurfaceZ of one die at n points, on the device (the queries the increment uses)
    void die_query(int side, int n, const double *p, double offset, double *clr, double *proj, double *nrm, double *sz)
    {
        if (side < 0 || side > 1 || !(have_dies & (1 << side))) throw Failure(IFEA_BAD_STATE, "that die is not set");
        if (n == 0) return;
        DBuf<double> dp, dout;
        dp.upload(p, 3 * (size_t)n, st);
        dout.resize(8 * (size_t)n);
        k_die_query<<<grid(n), 256, 0, st>>>(die[side], n, dp.p, offset, dout.p);
        cuda_check(cudaGetLastError(), "k_die_query");
        std::vector<double> o(8 * (size_t)n);
        dout.download(o.data(), o.size(), st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        for (int i = 0; i < n; i++) {
            clr[i] = o[8 * (size_t)i];
            for (int a = 0; a < 3; a++) proj[3 * (size_t)i + a] = o[8 * (size_t)i + 1 + a], nrm[3 * (size_t)i + a] = o[8 * (size_t)i + 4 + a];
            sz[i] = o[8 * (size_t)i + 7];
        }
    }

    void set_die(int side, int nx, int ny, double x0, double y0, double dx, const double *hh)
    {
        if (side < 0 || side > 1 || nx < 1 || ny < 1 || !(dx > 0)) throw Failure(IFEA_INPUT_INVALID, "invalid die grid");
        die_h[side].upload(hh, (size_t)(nx + 1) * (ny + 1), st);
        die_host[side].assign(hh, hh + (size_t)(nx + 1) * (ny + 1));
        die[side].side = side; die[side].nx = nx; die[side].ny = ny;
        die[side].x0 = x0; die[side].y0 = y0; die[side].dx = dx; die[side].h = die_h[side].p;
        die[side].kind = 0;
        have_dies |= 1 << side;
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }

    double volume()
    {
        View3 V = view();
        k_volume<<<kReduceBlocks, 256, 0, st>>>(V);
        finalize({S_VOLUME});
        return read_scalars()[S_VOLUME] * P.sym_factor;
    }

    // Constructor tail (Forging3DSolver.cs:156-184)
    void init(double g0, double min_x, double min_y, double min_z, double max_x, double max_y)
    {
        if (have_dies != 3 || topo.nn == 0) throw Failure(IFEA_INPUT_INVALID, "mesh and both dies must be set first");
        gap0 = gap = g0;
        View3 V = view();
        int nn = topo.nn;
        std::vector<double> cb(nn), ct(nn);
        d_pred.resize(3 * (size_t)nn);
        k_initial_contact<<<grid(nn), 256, 0, st>>>(V, 0.05 * h, d_pred.p, d_pred.p + nn);
        std::vector<uint8_t> contact(nn);
        d_contact.download(contact.data(), nn, st);
        cuda_check(cudaMemcpyAsync(cb.data(), d_pred.p, nn * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaMemcpyAsync(ct.data(), d_pred.p + nn, nn * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        int nb = 0, ntop = 0;
        for (int n = 0; n < nn; n++) { nb += contact[n] == IFEA_BOTTOM_DIE; ntop += contact[n] == IFEA_TOP_DIE; }
        // ForceContact (:366-378): the surface node with the smallest clearance, first on ties
        auto force = [&](int side, const std::vector<double> &c) {
            int best = -1;
            double bc = DBL_MAX;
            for (int n = 0; n < nn; n++)
                if (topo.is_surface[n] && c[n] < bc) { bc = c[n]; best = n; }
            if (best >= 0) contact[best] = (uint8_t)side;
        };
        if (nb == 0) force(IFEA_BOTTOM_DIE, cb);
        if (ntop == 0) force(IFEA_TOP_DIE, ct);
        d_contact.upload(contact, st);
        k_place_and_velocity<<<grid(nn), 256, 0, st>>>(V, rate_ref, 0, 0, 0);
        k_initial_velocity<<<grid(nn), 256, 0, st>>>(V, rate_ref, 0.5 * (min_x + max_x), 0.5 * (min_y + max_y), min_z);
        vol0 = volume();
        initialized = true;
    }

    // ---------------------------------------------------------------- PrepareStep (:660-758)
    void prepare_step()
    {
        PhaseTimer pt(t_prepare);
        View3 V = view();
        reset_err();
        k_frames<<<grid(topo.nn), 256, 0, st>>>(V);
        k_grad<<<grid(topo.ne), 256, 0, st>>>(V);
        int32_t e4[4];
        read_err(e4);
        if (e4[0] != INT_MAX) throw Failure(IFEA_MESH_DISTORTED, fmt("Tetrahedron %d is inverted at step %d.", e4[0], step_index));
        k_anp_coef<<<grid(topo.nn), 256, 0, st>>>(V);
        int G = (int)topo.g_node.size();
        k_clocal<<<grid(G), 256, 0, st>>>(V, G);
        k_kvol<<<std::min(kReduceBlocks * 2, (topo.nn + wpb - 1) / wpb), wpb * 32, col_smem, st>>>(V, topo.max_nbr);
        k_friction_prep<<<grid(topo.nn), 256, 0, st>>>(V);
        int trend = P.extrapolate_start && warm && have_vg_prev;
        k_guess<<<grid(topo.nn), 256, 0, st>>>(V, trend);
        cuda_check(cudaGetLastError(), "prepare_step launch");
        if (ws_net && ws_mode) warm_start_guess();
    }

    void warm_start_guess()
    {
        int nn = topo.nn;
        d_wsf.resize((size_t)16 * nn);
        d_wsv0.resize((size_t)3 * nn);
        View3 V = view();
        k_ws_features<<<grid(nn), 256, 0, st>>>(V, d_wsf, d_wsv0, rate_ref, h, P.ds, P.size, have_vg_prev ? 1 : 0);
        if (!(ws_mode & 2) || !warm || !have_vg_prev) return;
        d_wsy.resize((size_t)3 * nn);
        ws_net->infer_device(d_wsf, nn, d_wsy, st);
        if (ws_smooth > 0) {
            d_wsy2.resize((size_t)3 * nn);
            for (int p = 0; p < ws_smooth; p++) {
                k_ws_smooth<<<grid(nn), 256, 0, st>>>(V, d_wsy, d_wsy2);
                swap_buf(d_wsy, d_wsy2);
            }
        }
        k_ws_guess<<<grid(nn), 256, 0, st>>>(V, d_wsv0, d_wsy, d_vbuf[1 - vcur]);
        if (ws_policy == 1) {  // the network's start, unconditionally
            vcur = 1 - vcur;
            ws_used++;
            return;
        }
        // the Newton iteration minimises the functional: measure the starts by it
        double e_ref = assemble(ASM_ENERGY, 0, d_vbuf[vcur], false, nullptr);
        double e_net = assemble(ASM_ENERGY, 0, d_vbuf[1 - vcur], false, nullptr);
        if (ws_policy == 0) {  // whichever start has the lower value
            if (e_net < e_ref) {
                vcur = 1 - vcur;
                ws_used++;
            } else {
                ws_fallbacks++;
            }
            return;
        }
        // policy 2: the prediction as a search direction from the reference start, v(a) = v_ref + a (v_net - v_ref),
        // with the step from a parabola through a = 0, 1/2, 1 (clamped to [0, 1.5]); the lowest of the tried
        // points is kept, so the reference start (a = 0) stays the fallback
        int n = topo.ndof;
        d_wstry.resize((size_t)n);
        const double *v0 = d_vbuf[vcur], *v1 = d_vbuf[1 - vcur];
        k_ws_mix<<<grid(n), 256, 0, st>>>(n, v0, v1, 0.5, d_wstry);
        double e_half = assemble(ASM_ENERGY, 0, d_wstry, false, nullptr);
        double c2 = 2 * (e_ref - 2 * e_half + e_net), c1 = e_net - e_ref - c2;  // e(a) = e_ref + c1 a + c2 a^2
        double best_a = 0, best_e = e_ref;
        if (e_half < best_e) { best_a = 0.5; best_e = e_half; }
        if (e_net < best_e) { best_a = 1.0; best_e = e_net; }
        if (c2 > 0) {
            double a = rclamp(-c1 / (2 * c2), 0.0, 1.5);
            if (a != 0 && a != 0.5 && a != 1.0) {
                k_ws_mix<<<grid(n), 256, 0, st>>>(n, v0, v1, a, d_wstry);
                double e_a = assemble(ASM_ENERGY, 0, d_wstry, false, nullptr);
                if (e_a < best_e) { best_a = a; best_e = e_a; }
            }
        }
        ws_last_step = best_a;
        if (best_a == 0) {
            ws_fallbacks++;
            return;
        }
        ws_used++;
        if (best_a == 1.0) {
            vcur = 1 - vcur;
            return;
        }
        k_ws_mix<<<grid(n), 256, 0, st>>>(n, v0, v1, best_a, d_vbuf[1 - vcur]);
        vcur = 1 - vcur;
    }

    void warm_start_record()
    {
        if (!ws_net || !(ws_mode & 1) || d_wsv0.n != (size_t)3 * topo.nn) return;
        d_wst.resize((size_t)3 * topo.nn);
        View3 V = view();
        k_ws_targets<<<grid(topo.nn), 256, 0, st>>>(V, d_wsv0, d_wst);
        ws_net->add_samples_device(d_wsf, d_wst, topo.nn, st);
    }

    // ---------------------------------------------------------------- Assemble (:1115-1217)
    // Returns energy; power via *pw. bc: apply the BC pass inside the column kernel (MATRIX only).
    double assemble(int mode, int newton, const double *v, bool bc, double *pw)
    {
        n_assemble++;
        View3 V = view();
        switch (mode) {
        case ASM_MATRIX: k_element<ASM_MATRIX><<<kReduceBlocks, 256, 0, st>>>(V, v, newton); break;
        case ASM_RESIDUAL: k_element<ASM_RESIDUAL><<<kReduceBlocks, 256, 0, st>>>(V, v, newton); break;
        default: k_element<ASM_ENERGY><<<kReduceBlocks, 256, 0, st>>>(V, v, newton); break;
        }
        int cb = kReduceBlocks;
        if (mode == ASM_MATRIX && bc) k_columns<ASM_MATRIX, true><<<cb, wpb * 32, col_smem, st>>>(V, v, newton, topo.max_nbr);
        else if (mode == ASM_MATRIX) k_columns<ASM_MATRIX, false><<<cb, wpb * 32, col_smem, st>>>(V, v, newton, topo.max_nbr);
        else if (mode == ASM_RESIDUAL) k_columns<ASM_RESIDUAL, false><<<cb, wpb * 32, 0, st>>>(V, v, newton, topo.max_nbr);
        else k_columns<ASM_ENERGY, false><<<cb, wpb * 32, 0, st>>>(V, v, newton, topo.max_nbr);
        cuda_check(cudaGetLastError(), "assemble launch");
        finalize({S_E_VOL, S_E_ELEM, S_E_FRIC, S_P_ELEM, S_P_FRIC, S_RNORM2, MAXS(S_MAXDIAG)});
        const double *s = read_scalars();
        double energy = s[S_E_VOL] + s[S_E_ELEM] + s[S_E_FRIC];
        if (pw) *pw = 2 * s[S_E_VOL] + s[S_P_ELEM] + s[S_P_FRIC];
        if (mode == ASM_MATRIX && bc) {
            max_diag = s[S_MAXDIAG];
            rnorm = sqrt(s[S_RNORM2]);
        }
        return energy;
    }

    void apply_bc_separately()
    {
        View3 V = view();
        k_apply_bc<<<kReduceBlocks, 256, 0, st>>>(V);
        finalize({MAXS(S_MAXDIAG)});
        k_regularise<<<grid(topo.ndof), 256, 0, st>>>(V);
        max_diag = read_scalars()[S_MAXDIAG];
    }

    // ---------------------------------------------------------------- SolveLinear (:965-1019) and Pcg (:1051-1087)
    double dot_read(const double *a, const double *b, int slot, const double *c = nullptr, int slot2 = S_NORM_B,
                    double *second = nullptr)
    {
        View3 V = view();
        k_dot2<<<kReduceBlocks, 256, 0, st>>>(V, a, b, slot, c, slot2);
        if (c) finalize({slot, slot2}); else finalize({slot});
        const double *s = read_scalars();
        if (second) *second = s[slot2];
        return s[slot];
    }

    int pcg(const double *b, double *x, double tol, int max_it)
    {
        View3 V = view();
        int n = topo.ndof;
        double bb = dot_read(b, b, S_BB);
        double bnorm = sqrt(bb);
        if (bnorm == 0) {
            cuda_check(cudaMemsetAsync(x, 0, n * sizeof(double), st), "memset");
            return 0;
        }
        int sp_grid = std::min(kReduceBlocks * 4, (topo.nn * 32 + 255) / 256);
        lin->solve(b, x);
        k_spmv<<<sp_grid, 256, 0, st>>>(V, x, d_pq);
        k_pcg_residual<<<grid(n), 256, 0, st>>>(n, b, d_pq, d_pr);
        lin->solve(d_pr, d_pz);
        cuda_check(cudaMemcpyAsync(d_pp.p, d_pz.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st), "D2D");
        k_dot2<<<kReduceBlocks, 256, 0, st>>>(V, d_pr, d_pz, S_RZ, d_pr, S_RR);
        finalize({S_RZ, S_RR});
        double rr = read_scalars()[S_RR];
        double r0 = sqrt(rr);
        for (int it = 0; it < max_it; it++) {
            if (sqrt(rr) <= tol * bnorm) return it;
            if (pcg_early_abort && it >= 3) {
                // the observed contraction cannot reach the tolerance within the budget: refactorise now
                double rate = pow(sqrt(rr) / r0, 1.0 / it);
                if (!(rate < 1) || it + log(tol * bnorm / sqrt(rr)) / log(rate) > max_it) return -1;
            }
            k_spmv<<<sp_grid, 256, 0, st>>>(V, d_pp, d_pq);
            k_dot2<<<kReduceBlocks, 256, 0, st>>>(V, d_pp, d_pq, S_PQ, nullptr, 0);
            finalize({S_PQ});
            k_pcg_xr<<<grid(n), 256, 0, st>>>(n, d_scalars, x, d_pr, d_pp, d_pq);
            lin->solve(d_pr, d_pz);
            k_dot2<<<kReduceBlocks, 256, 0, st>>>(V, d_pr, d_pz, S_RZNEW, d_pr, S_RR);
            finalize({S_RZNEW, S_RR});
            k_pcg_p<<<grid(n), 256, 0, st>>>(n, d_scalars, d_pp, d_pz);
            k_pcg_roll<<<1, 1, 0, st>>>(d_scalars);
            rr = read_scalars()[S_RR];
            lin_its++;
        }
        return sqrt(rr) <= tol * bnorm ? max_it : -1;
    }

    // PCG iterations a reused factor may take. The reference's budget (PcgBudget, 15) in the FP64 form; in the
    // single-precision form, whose factorisations are measured (device time) as are its PCG iterations (host
    // time, syncs included), a reused factor is worth iterations up to pcg_budget_scale factorisations' time
    // (at least the reference's budget, at most 120)
    int pcg_budget()
    {
        if (!pcg_early_abort || n_fact == 0 || lin_its == 0) return P.pcg_budget;
        double f_ms = lin->factor_ms() / n_fact, it_ms = 1000.0 * t_pcg / lin_its;
        if (!(f_ms > 0) || !(it_ms > 0)) return P.pcg_budget;
        return std::max(P.pcg_budget, std::min(120, (int)(pcg_budget_scale * f_ms / it_ms)));
    }

    // b -> x; returns 0 for PCG, 1 for a fresh factorisation
    int solve_linear(const double *b, double *x)
    {
        // single-precision form: a factor from an earlier increment is tried again only every eighth increment
        // once such a try has failed (tries within the increment of the factor are unaffected)
        bool stale = have_factor && factor_step != step_index;
        bool skip_stale = pcg_early_abort && stale && stale_failures > 0 && step_index % 8 != 0;
        if (have_factor && pcg_skip > 0) {
            pcg_skip--;
        } else if (have_factor && !skip_stale) {
            int its;
            {
                PhaseTimer pt(t_pcg);
                its = pcg(b, x, lin_tol, pcg_budget());
            }
            if (stale) stale_failures = its >= 0 ? 0 : stale_failures + 1;
            if (its >= 0) {
                pcg_failures = 0;
                n_pcg++;
                return 0;
            }
            pcg_failures_total++;
            if (++pcg_failures >= 2) pcg_skip = std::min(64, 1 << (pcg_failures - 1));
        }
        if (need_analyze) {
            analyze_pattern();
            need_analyze = false;
        }
        try {
            PhaseTimer pt(t_factor);
            try {
                lin->factorize(d_val);
            } catch (Failure &f) {
                // a pivot lost to single-precision rounding: continue in double precision for good
                if (f.status != IFEA_NOT_SPD || lin->value_bytes() == 8) throw;
                use_precision(false);
                fp32_fallbacks++;
                lin->analyze(topo.ndof, topo.col_ptr.data(), topo.row_idx.data(), 3,
                             ordering == 1 ? node_xyz.data() : nullptr);
                need_analyze = false;
                lin->factorize(d_val);
            }
            if (lin->value_bytes() == 8) {
                lin->solve(b, x);
                lin->check_finite(x);
            }
        } catch (Failure &f) {
            have_factor = false;
            if (f.status == IFEA_NOT_SPD) throw;
            throw Failure(IFEA_DIVERGED, fmt("Sparse factorisation failed at step %d (GPU multifrontal Cholesky): %s", step_index, f.what()));
        }
        have_factor = true;
        factor_step = step_index;
        n_fact++;
        if (lin->value_bytes() != 8) {
            // FP64 refinement of the single-precision factor's solution, to the tolerance of the reused-factor PCG
            PhaseTimer pt(t_pcg);
            int l0 = lin_its;
            int its = pcg(b, x, lin_tol, P.pcg_budget);
            refine_its += lin_its - l0;
            if (its < 0) {
                have_factor = false;
                throw Failure(IFEA_DIVERGED, fmt("Refinement of the single-precision factor did not converge at step %d.", step_index));
            }
        }
        return 1;
    }

    // ---------------------------------------------------------------- SolveVelocity (:875-948)
    int solve_velocity(bool *converged, const volatile int32_t *cancel)
    {
        *converged = false;
        last_rel = INFINITY;
        int it, halved = 0;
        bool secant_only = false;
        const int newton_limit = 20;
        int n = topo.ndof;
        for (it = 1; it <= P.max_iter; it++) {
            if (cancel && *cancel) throw Failure(IFEA_CANCELLED, "The operation was canceled.");
            if (P.sticky_secant && halved >= 2) secant_only = true;
            int newton = (warm || it > 2) && it <= newton_limit && !secant_only && !(P.adaptive_newton && halved >= 2);
            n_newton += newton;
            double e0;
            {
                PhaseTimer pt(t_assemble);
                e0 = assemble(ASM_MATRIX, newton, d_vbuf[vcur], true, nullptr);
            }
            {
                View3 V = view();
                k_regularise<<<grid(n), 256, 0, st>>>(V);
            }
            lin_tol = pcg_forcing > 0 ? rclamp(pcg_forcing * last_rel, 1e-7, 1e-3) : 1e-7;
            solve_linear(d_b, d_dv);
            // slope = sum R.dv with R fixed-zeroed (= -b.dv), and |dv|^2
            double dvdv = 0;
            double slope = -dot_read(d_b, d_dv, S_DOT, d_dv, S_NORM_B, &dvdv);
            double beta = 1;
            PhaseTimer pls(t_linesearch);
            for (int ls = 0; ls < 8; ls++) {
                k_axpy<<<grid(n), 256, 0, st>>>(n, d_vbuf[1 - vcur], d_vbuf[vcur], d_dv, beta);
                double e1 = assemble(ASM_ENERGY, 0, d_vbuf[1 - vcur], false, nullptr);
                if (e1 <= e0 + 1e-4 * beta * slope + 1e-11 * fabs(e0)) break;
                double curv = (e1 - e0 - slope * beta) / (beta * beta);
                beta = P.quadratic_ls && curv > 0 ? rclamp(-slope / (2 * curv), 0.1 * beta, 0.7 * beta) : 0.5 * beta;
            }
            vcur = 1 - vcur;
            halved = newton && beta < 1 ? halved + 1 : 0;
            double vv = dot_read(d_vbuf[vcur], d_vbuf[vcur], S_NORM_A);
            double rel = beta * sqrt(dvdv) / rmax(sqrt(vv), 1e-30);
            last_rel = rel;
            beta_last = beta;
            if (std::isnan(rel)) throw Failure(IFEA_DIVERGED, fmt("Velocity solution became NaN at step %d.", step_index));
            if (rel < P.tol) {
                *converged = true;
                return it;
            }
        }
        return it - 1;
    }

    // ---------------------------------------------------------------- FinalEvaluation (:1402-1451)
    double final_evaluation(double *reaction_out)
    {
        PhaseTimer pt(t_final);
        double pw = 0;
        assemble(ASM_RESIDUAL, 0, d_vbuf[vcur], false, &pw);
        View3 V = view();
        k_final_nodes<<<kReduceBlocks, 256, 0, st>>>(V);
        finalize({S_REACTION, MAXS(S_MAX_B), MAXS(S_MAX_T)});
        k_release<<<kReduceBlocks, 256, 0, st>>>(V);
        finalize({S_KEPT_B, S_KEPT_T});
        k_release_keep<<<grid(topo.nn), 256, 0, st>>>(V);
        k_nodal_mean<<<grid(topo.nn), 256, 0, st>>>(V, d_nodal);
        k_el_mean<<<grid(topo.ne), 256, 0, st>>>(V, d_nodal);
        const double *s = read_scalars();
        have_vg_prev = true;
        reaction = s[S_REACTION];
        if (reaction_out) *reaction_out = reaction;
        power = pw;
        return pw;
    }

    // ---------------------------------------------------------------- TryUpdate (:1455-1537)
    double min_quality(const double *x)
    {
        View3 V = view();
        k_quality_check<<<kReduceBlocks, 256, 0, st>>>(V, x, -INFINITY);
        finalize({MAXS(S_MINQ)});
        return -read_scalars()[S_MINQ];
    }

    int smooth_interior(double *x, double qtarget, int sweeps)
    {
        View3 V = view();
        d_counters.zero(st);
        k_smooth_interior<<<1, 32, 0, st>>>(V, x, qtarget, sweeps, d_bad, d_counters.p + 2);
        int32_t c[4];
        d_counters.download(c, 4, st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        return c[2];
    }

    bool try_update(double dt, std::string &why)
    {
        PhaseTimer pt(t_update);
        double gapT = rmax(0, gap - P.ram * dt);
        if (gapT < 1e-9) gapT = 0;
        View3 V = view();
        int nn = topo.nn;
        bool lenient = recovery_pass >= 2;
        k_surface_normals<<<grid(nn), 256, 0, st>>>(V, d_x, d_nrm);
        k_predict<<<kReduceBlocks, 256, 0, st>>>(V, dt, gapT, h, lenient, d_xT, d_pred, d_cT);
        finalize({MAXS(S_MAXPEN)});
        double maxPenRel = read_scalars()[S_MAXPEN];
        if (maxPenRel > 0.5) {
            why = "die penetration exceeds half the local element size";
            return false;
        }
        if (min_quality(d_xT) < 0.05) {
            static const double ladder[2] = {0.05, 0.1};
            double frac = ladder[iclamp(recovery_pass, 0, 1)];
            d_counters.zero(st);
            k_improve_placement<<<1, 32, 0, st>>>(V, d_xT, d_cT, d_pred, d_nrm, gapT, 0.05, h, lenient, frac, d_counters);
            int32_t c[4];
            d_counters.download(c, 4, st);
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            projection_reverts += c[0];
            corner_penetrations += c[1];
            if (min_quality(d_xT) < 0.05) smooth_interior(d_xT, 0.05, 6);
        }
        reset_err();
        k_quality_check<<<kReduceBlocks, 256, 0, st>>>(V, d_xT, 0.005);
        int32_t e4[4];
        read_err(e4);
        if (e4[1] != INT_MAX) {
            why = fmt("tetrahedron %d collapsed", e4[1]);
            {
                // the failure point for local refinement at the next remesh: the collapsed tet's centroid
                double xt[12];
                for (int a = 0; a < 4; a++)
                    cuda_check(cudaMemcpyAsync(xt + 3 * a, d_xT.p + 3 * (size_t)topo.tets[4 * (size_t)e4[1] + a],
                                               3 * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
                cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
                fail_at = mk3(0.25 * (xt[0] + xt[3] + xt[6] + xt[9]), 0.25 * (xt[1] + xt[4] + xt[7] + xt[10]),
                              0.25 * (xt[2] + xt[5] + xt[8] + xt[11]));
                have_fail_at = true;
            }
            return false;
        }
        swap_buf(d_x, d_xT);
        swap_buf(d_contact, d_cT);
        gap = gapT;
        time += dt;
        return true;
    }

    // one factorisation of the current (assembled, constrained) matrix and one solve, device milliseconds: the
    // measurement the launch-parameter tuner compares (ifea3d_autotune)
    double time_factor_solve()
    {
        if (need_analyze) {
            analyze_pattern();
            need_analyze = false;
        }
        cudaEvent_t a, b;
        cuda_check(cudaEventCreate(&a), "cudaEventCreate");
        cuda_check(cudaEventCreate(&b), "cudaEventCreate");
        cuda_check(cudaEventRecord(a, st), "cudaEventRecord");
        lin->factorize(d_val);
        lin->solve(d_r, d_dv);
        cuda_check(cudaEventRecord(b, st), "cudaEventRecord");
        cuda_check(cudaEventSynchronize(b), "cudaEventSynchronize");
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        have_factor = true;
        factor_step = step_index;
        return ms;
    }

    // ---------------------------------------------------------------- FillPercent (:2149-2189)
    void set_cavity(int n, const double *xyz)
    {
        if (n < 0 || (n > 0 && !xyz)) throw Failure(IFEA_INPUT_INVALID, "invalid cavity samples");
        d_cavity.upload(xyz, 3 * (size_t)n, st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    }

    double fill_percent()
    {
        int np = (int)(d_cavity.n / 3);
        if (np == 0) return 0;
        View3 V = view();
        k_node_box<<<kReduceBlocks, 256, 0, st>>>(V);
        finalize({MAXS(S_BOX0), MAXS(S_BOX1), MAXS(S_BOX2), MAXS(S_BOX3), MAXS(S_BOX4), MAXS(S_BOX5)});
        const double *b = read_scalars();
        LocGrid G;
        G.cell = 2 * h;
        G.x0 = -b[S_BOX3] - G.cell; G.y0 = -b[S_BOX4] - G.cell; G.z0 = -b[S_BOX5] - G.cell;
        G.nx = (int)((b[S_BOX0] - G.x0) / G.cell) + 2;
        G.ny = (int)((b[S_BOX1] - G.y0) / G.cell) + 2;
        G.nz = (int)((b[S_BOX2] - G.z0) / G.cell) + 2;
        int ncell = G.nx * G.ny * G.nz;
        d_loc_start.resize(ncell + 1);
        d_loc_fill.resize(ncell + 1);
        d_loc_start.zero(st);
        k_loc_tets<<<grid(topo.ne), 256, 0, st>>>(V, G, 0, d_loc_start, nullptr, nullptr);
        k_scan_block<<<1, 1024, 0, st>>>(d_loc_start, ncell + 1, d_loc_fill);
        int32_t total = 0;
        cuda_check(cudaMemcpyAsync(&total, d_loc_start.p + ncell, sizeof total, cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        d_loc_items.resize(std::max(total, 1));
        k_loc_tets<<<grid(topo.ne), 256, 0, st>>>(V, G, 1, nullptr, d_loc_fill, d_loc_items);
        k_fill_query<<<kReduceBlocks, 256, 0, st>>>(V, G, d_loc_start, d_loc_items, d_cavity, np);
        finalize({S_FILL});
        return 100.0 * read_scalars()[S_FILL] / np;
    }

    // ---------------------------------------------------------------- Remesh (:1945-2101)
    bool remesh(const std::string &reason)
    {
        PhaseTimer pt(t_remesh);
        if (have_dies != 3) throw Failure(IFEA_BAD_STATE, "remeshing needs both dies");
        size_t nn = topo.nn, ne = topo.ne;
        std::vector<double> x(3 * nn), vg(3 * nn), eps(ne), dmg(ne), sig(ne), rate(ne), mean(ne);
        d_x.download(x.data(), 3 * nn, st);
        d_vg.download(vg.data(), 3 * nn, st);
        d_eps.download(eps.data(), ne, st);
        d_dmg.download(dmg.data(), ne, st);
        d_elsig.download(sig.data(), ne, st);
        d_elrate.download(rate.data(), ne, st);
        d_elmean.download(mean.data(), ne, st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        RemeshInput in;
        in.nn = (int)nn; in.ne = (int)ne; in.x = x.data(); in.tets = topo.tets.data(); in.vg = vg.data();
        in.eps = eps.data(); in.dmg = dmg.data(); in.sig = sig.data(); in.rate = rate.data(); in.mean = mean.data();
        for (int k = 0; k < 2; k++) {
            in.die[k] = die[k];
            if (die[k].kind == 1) in.die[k].tm = tm_host[k].grid;  // host copies of the grids
            else in.die[k].h = die_host[k].data();
        }
        in.gap = gap; in.h = h; in.vol_target = vol0 / P.sym_factor; in.sym_x = P.sym_x != 0; in.sym_y = P.sym_y != 0;
        in.recovery_pass = recovery_pass; in.refinement_levels = refinement_levels; in.max_nodes = max_nodes;
        in.sig_ref = sig_ref; in.hot = hot;
        in.on_topology = [this](const std::vector<d3> &px, const std::vector<int32_t> &pt, const std::vector<uint8_t> &onx,
                                const std::vector<uint8_t> &ony) { start_ahead(px, pt, onx, ony); };
        RemeshOutput out;
        if (!remesh_workpiece(in, out)) {
            remesh_rejected++;
            last_remesh = reason + " rejected: " + out.why;
            return false;
        }
        t_rm_stuff += out.t_stuff;
        t_rm_refine += out.t_refine;
        t_rm_place += out.t_place;
        t_rm_remap += out.t_remap;
        int nn2 = (int)(out.x.size() / 3), ne2 = (int)(out.tets.size() / 4);
        PhaseTimer pm(t_rm_setmesh);
        set_mesh(nn2, ne2, out.x.data(), out.tets.data(), out.on_x0.data(), out.on_y0.data());
        d_vg.upload(out.vg, st);
        d_eps.upload(out.eps, st);
        d_dmg.upload(out.dmg, st);
        d_elsig.upload(out.sig, st);
        d_elrate.upload(out.rate, st);
        d_elmean.upload(out.mean, st);
        d_contact.upload(out.contact, st);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        have_vg_prev = false;
        warm = 0;
        factor_step = -1;
        remesh_count++;
        last_remesh = fmt("%s: q_min %.3f -> %.3f, %d tets, %d nodes, %d local refinements", reason.c_str(), out.q_old,
                          out.q_new, ne2, nn2, out.splits);
        return true;
    }

    // ---------------------------------------------------------------- Step (:540-638)
    void step(ifea_step_info *info, const volatile int32_t *cancel)
    {
        if (!initialized) throw Failure(IFEA_BAD_STATE, "ifea3d_init must be called before stepping.");
        if (gap <= 1e-9) throw Failure(IFEA_BAD_STATE, "Simulation already reached the closed-die position.");
        step_index++;
        PhaseTimer ptotal(t_total);
        // RemeshTrigger (:1867-1883): first-aid smoothing; a remesh itself is out of scope and only counted
        {
            PhaseTimer pt(t_trigger);
            double rq = P.remesh_quality;
            const char *trigger = nullptr;
            if (min_quality(d_x) < rq) smooth_interior(d_x, rq, 6);
            if (min_quality(d_x) < rq) trigger = "element quality";
            else {
                View3 V = view();
                k_edges_layers<<<kReduceBlocks, 256, 0, st>>>(V);
                finalize({MAXS(S_MAXEDGE), MAXS(S_THIN)});
                if (read_scalars()[S_MAXEDGE] > 2.8 * h) trigger = "surface stretched";
            }
            if (trigger) {
                remesh_requests++;
                if (remesh_enabled) remesh(trigger);
            }
        }
        double step_cap = P.ds * h / P.h;
        int its = 0, used_cutback = 0;
        bool ok = false;
        double dt = 0;
        std::string why;
        const int passes = 4;
        for (int pass = 0; pass < passes && !ok; pass++) {
            recovery_pass = pass;
            prepare_step();
            bool converged = false;
            its = solve_velocity(&converged, cancel);
            if (!converged) {
                if (!(last_rel < 1e-2)) {
                    if (pass < passes - 1) {
                        remesh_requests++;
                        if (remesh_enabled && remesh("stalled velocity solution")) continue;
                    }
                    throw Failure(IFEA_DIVERGED, fmt("Velocity solution did not converge at step %d (stroke %.3f mm): |dv|/|v| = %.2e.",
                                                     step_index, gap0 - gap, last_rel));
                }
            }
            double pw = final_evaluation(&reaction);
            load = pw / P.ram * P.sym_factor;
            reaction *= P.sym_factor;
            View3 V = view();
            k_edges_layers<<<kReduceBlocks, 256, 0, st>>>(V);
            finalize({MAXS(S_MAXEDGE), MAXS(S_THIN)});
            double thin_neg = read_scalars()[S_THIN];
            double thinnest = std::isfinite(thin_neg) ? -thin_neg : INFINITY;
            double layer = std::isfinite(thinnest) ? rmax(0.1 * thinnest, step_cap / (1 << P.max_cutbacks)) : INFINITY;
            double ds = rmin(P.auto_step ? rmin(ds_cur, step_cap) : step_cap, layer);
            dt = rmin(ds, gap) / P.ram;
            if (gap - P.ram * dt < 0.05 * ds) dt = gap / P.ram;
            for (int attempt = 0; attempt <= P.max_cutbacks && !ok; attempt++) {
                double dta = dt / (1 << attempt);
                ok = try_update(dta, why);
                if (ok) {
                    dt = dta;
                    used_cutback = attempt;
                }
            }
            if (ok || pass == passes - 1) break;
            if (pass >= 1 && refinement_levels > 0 && have_fail_at) {
                hot.push_back({fail_at, std::min(pass, refinement_levels)});
                if (hot.size() > 64) hot.erase(hot.begin());
            }
            remesh_requests++;
            // a rejected remesh does not end the ladder: the next pass relaxes the corner tolerance
            if (remesh_enabled) remesh(pass == 0 ? "fold during update" : "recovery");
        }
        recovery_pass = 0;
        if (!ok)
            throw Failure(IFEA_MESH_DISTORTED, fmt("Mesh distortion at step %d (stroke %.3f mm): %s. Automatic cutbacks, remeshing and local refinement could not recover.",
                                                   step_index, gap0 - gap, why.c_str()));
        if (P.auto_step) {
            double used = P.ram * dt;
            ds_cur = used_cutback > 0 ? rmax(used, step_cap / (1 << P.max_cutbacks)) : rmin(step_cap, 1.5 * ds_cur);
        }
        warm_start_record();
        View3 V = view();
        k_strain_damage<<<grid(topo.ne), 256, 0, st>>>(V, dt);
        warm = 1;
        iterations = its;
        last_cutbacks = used_cutback;
        last_dt = dt;
        double vol = volume();
        if (info) {
            info->step = step_index;
            info->iterations = its;
            info->load = load;
            info->reaction = reaction;
            info->stroke = gap0 - gap;
            info->gap = gap;
            info->time = time;
            info->dt = dt;
            info->volume_change_pct = 100.0 * (vol - vol0) / vol0;
            info->last_rel = last_rel;
            info->n_factor = n_fact;
            info->n_pcg = n_pcg;
            info->remesh_requests = remesh_requests;
            info->cutbacks = used_cutback;
        }
    }

    // ---------------------------------------------------------------- array access
    struct ArrRef {
        void *p;
        size_t count;
        int bytes;
    };
    ArrRef array(const std::string &nm)
    {
        size_t nn = topo.nn, ne = topo.ne, nd = topo.ndof;
#define A(name, buf, cnt) if (nm == name) return ArrRef{(void *)(buf).p, (size_t)(cnt), (int)sizeof(*(buf).p)};
        A("x", d_x, 3 * nn) A("vg", d_vg, 3 * nn) A("v", d_vbuf[vcur], nd) A("r", d_r, nd) A("dv", d_dv, nd) A("b", d_b, nd)
        A("eps", d_eps, ne) A("dmg", d_dmg, ne) A("el_sig", d_elsig, ne) A("el_rate", d_elrate, ne)
        A("el_mean", d_elmean, ne) A("el_dev", d_eldev, 6 * ne) A("grad", d_grad, 12 * ne) A("vol", d_vol, ne)
        A("ax", d_ax, 9 * nn) A("fixed_val", d_fixedval, nd) A("k_fric", d_kfric, nn) A("a_fric", d_afric, nn)
        A("v_node", d_vnode, nn) A("kvol", d_kvol, topo.nnz) A("val", d_val, topo.nnz) A("h_local", d_hloc, nn)
        A("contact", d_contact, nn) A("release", d_release, nn) A("fixed", d_fixed, nd) A("n_fix", d_nfix, nn)
        A("die_axis", d_dieaxis, nn) A("nbr_start", d_nbr_start, nn + 1) A("nbr", d_nbr, topo.nbr.size())
        A("e_r", d_er, 12 * ne) A("g_coef", d_gcoef, 3 * topo.g_node.size()) A("g_node", d_gnode, topo.g_node.size())
        A("g_start", d_gstart, nn + 1) A("vg_prev", d_vgprev, 3 * nn) A("tets", d_tets, 4 * ne)
#undef A
        if (nm == "e_nbr") return ArrRef{(void *)topo.e_nbr.data(), topo.e_nbr.size(), -4};
        if (nm == "bface") return ArrRef{(void *)topo.bface.data(), topo.bface.size(), -4};
        if (nm == "is_surface") return ArrRef{(void *)topo.is_surface.data(), topo.is_surface.size(), -1};
        throw Failure(IFEA_INPUT_INVALID, "unknown array name '" + nm + "'");
    }

    // floating-point operations of one factorisation of the current pattern: per front of m rows and k pivot
    // columns, the lower-triangle updates sum over c < k of (m - c - 1)(m - c) (a multiply and an add each), plus
    // the pivot column scalings
    double factor_gflop()
    {
        const MfSymbolic &S = lin->symbolic();
        double f = 0;
        for (int s = 0; s < S.nsuper; s++) {
            double m = S.m[s];
            for (int c = 0; c < S.ncol[s]; c++) f += (m - c - 1) * (m - c) + (m - c - 1);
        }
        return f * 1e-9;
    }

    double scalar(const std::string &nm)
    {
#define S(name, v) if (nm == name) return (double)(v);
        S("gap", gap) S("gap0", gap0) S("time", time) S("load", load) S("reaction", reaction) S("power", power)
        S("iterations", iterations) S("last_rel", last_rel) S("vol0", vol0) S("step_index", step_index)
        S("n_pcg", n_pcg) S("n_fact", n_fact) S("n_newton", n_newton) S("n_assemble", n_assemble)
        S("remesh_requests", remesh_requests) S("projection_reverts", projection_reverts)
        S("corner_penetrations", corner_penetrations) S("rate_ref", rate_ref) S("rate_cut", rate_cut)
        S("sig_ref", sig_ref) S("k_pen", k_pen) S("u0", u0) S("nnz", topo.nnz) S("ds_cur", ds_cur) S("warm", warm)
        S("rnorm", rnorm) S("beta", beta_last) S("max_diag", max_diag) S("have_factor", have_factor)
        S("pcg_skip", pcg_skip) S("pcg_failures", pcg_failures) S("lin_its", lin_its) S("nbf", topo.bowner.size())
        S("recovery_pass", recovery_pass) S("factor_nnz", lin->factor_nonzeros()) S("max_nbr", topo.max_nbr)
        S("nn", topo.nn) S("ne", topo.ne) S("ndof", topo.ndof) S("last_dt", last_dt)
        S("t_trigger", t_trigger) S("t_prepare", t_prepare) S("t_assemble", t_assemble) S("t_linesearch", t_linesearch)
        S("t_factor", t_factor) S("t_pcg", t_pcg) S("t_final", t_final) S("t_update", t_update) S("t_total", t_total)
        S("supernodes", lin->symbolic().nsuper) S("levels", lin->symbolic().nlevels)
        S("front_pool_mb", lin->symbolic().pool * lin->value_bytes() * 1e-6) S("max_front", lin->symbolic().max_m) S("big_fronts", lin->big_fronts())
        S("ordering", ordering) S("t_symbolic", lin->setup_s(0)) S("t_order", lin->symbolic().order_s) S("t_symbolic_wait", t_sym_wait) S("t_symbolic_dev", lin->setup_s(1)) S("t_graph_factor", lin->setup_s(2))
        S("t_graph_solve", lin->setup_s(3)) S("factor_gpu_ms", lin->factor_ms()) S("solve_gpu_ms", lin->solve_ms()) S("solves", lin->solves())
        S("factor_fp32", lin->value_bytes() == 4) S("fp32_fallbacks", fp32_fallbacks) S("refine_its", refine_its)
        S("pcg_early_abort", pcg_early_abort) S("pcg_failures_total", pcg_failures_total) S("wide_front_rows", wide_rows) S("tc_updates", lin->tc_launches())
        S("factor_gflop", factor_gflop())
        S("pcg_budget_now", pcg_budget()) S("pcg_budget_scale", pcg_budget_scale) S("pcg_forcing", pcg_forcing)
        S("ws_used", ws_used) S("ws_fallbacks", ws_fallbacks) S("ws_mode", ws_mode) S("ws_policy", ws_policy) S("ws_smooth", ws_smooth)
        S("ws_last_step", ws_last_step)
        S("remesh", remesh_enabled) S("remesh_count", remesh_count) S("remesh_rejected", remesh_rejected)
        S("t_remesh", t_remesh) S("t_rm_stuff", t_rm_stuff) S("t_rm_refine", t_rm_refine) S("t_rm_place", t_rm_place) S("t_rm_remap", t_rm_remap) S("t_rm_setmesh", t_rm_setmesh) S("refinement_levels", refinement_levels) S("max_nodes", max_nodes) S("hot_spots", hot.size())
#undef S
        if (nm == "volume") return volume();
        if (nm == "fill_percent") return fill_percent();
        if (nm == "min_quality") return min_quality(d_x);
        throw Failure(IFEA_INPUT_INVALID, "unknown scalar name '" + nm + "'");
    }
    void set_scalar(const std::string &nm, double v)
    {
        if (nm == "gap") gap = v;
        else if (nm == "recovery_pass") recovery_pass = (int)v;
        else if (nm == "ds_cur") ds_cur = v;
        else if (nm == "warm") warm = (int)v;
        else if (nm == "profile_solves") lin->set_profile(v != 0);
        else if (nm == "tc_update") lin->set_tc(v != 0, 1024);
        else if (nm == "tc_rows") lin->set_tc(true, (int)v);
        else if (nm == "wide_front_rows") {
            wide_rows = (int)v;
            lin->set_wide_rows(wide_rows);
            need_analyze = true;
            have_factor = false;
        } else if (nm == "factor_fp32") {
            use_precision(v != 0);
            pcg_early_abort = v != 0;
        } else if (nm == "pcg_early_abort") pcg_early_abort = v != 0;
        else if (nm == "pcg_budget_scale") {
            if (!(v > 0 && v <= 16)) throw Failure(IFEA_INPUT_INVALID, "pcg_budget_scale must lie in (0, 16]");
            pcg_budget_scale = v;
        }
        else if (nm == "pcg_forcing") {
            if (!(v >= 0 && v <= 1)) throw Failure(IFEA_INPUT_INVALID, "pcg_forcing must lie in [0, 1]");
            pcg_forcing = v;
        }
        else if (nm == "remesh") remesh_enabled = v != 0;
        else if (nm == "ws_smooth") ws_smooth = std::max(0, (int)v);
        else if (nm == "ws_policy") {
            if (v != 0 && v != 1 && v != 2) throw Failure(IFEA_INPUT_INVALID, "ws_policy: 0, 1 or 2");
            ws_policy = (int)v;
        }
        else if (nm == "refinement_levels") {
            if (v < 0 || v > 3) throw Failure(IFEA_INPUT_INVALID, "Refinement levels must be 0-3.");
            refinement_levels = (int)v;
        } else if (nm == "max_nodes") max_nodes = (int)v;
        else if (nm == "ordering") {
            if (v != 0 && v != 1) throw Failure(IFEA_INPUT_INVALID, "ordering: 0 (METIS) or 1 (coordinate nested dissection)");
            if ((int)v != ordering) {
                ordering = (int)v;
                if (topo.nn > 0) start_analysis();
                need_analyze = true;
                have_factor = false;
            }
        }
        else throw Failure(IFEA_INPUT_INVALID, "unknown scalar name '" + nm + "'");
    }
};

}  // namespace ifea

using ifea::Failure;
using ifea::Forging3D;

struct ifea3d {
    Forging3D *s;
};

template <typename F>
static ifea_status guarded(ifea3d *c, F &&f)
{
    if (!c || !c->s) return IFEA_INPUT_INVALID;
    try {
        f(*c->s);
        c->s->err.clear();
        return IFEA_OK;
    } catch (Failure &e) {
        c->s->err = e.what();
        return e.status;
    } catch (std::bad_alloc &) {
        c->s->err = "host out of memory";
        return IFEA_CUDA_ERROR;
    } catch (std::exception &e) {
        c->s->err = e.what();
        return IFEA_CUDA_ERROR;
    }
}

extern "C" {

ifea_status ifea3d_create(const ifea3d_params *params, ifea3d **out)
{
    if (!params || !out) return IFEA_INPUT_INVALID;
    *out = nullptr;
    if (!(params->ram > 0) || !(params->h > 0) || !(params->ds > 0) || !(params->size > 0) || params->max_iter < 1 ||
        params->sym_factor < 1)
        return IFEA_INPUT_INVALID;
    try {
        ifea3d *c = new ifea3d;
        c->s = new Forging3D(*params);
        *out = c;
        return IFEA_OK;
    } catch (Failure &e) {
        return e.status;
    } catch (...) {
        return IFEA_CUDA_ERROR;
    }
}

void ifea3d_destroy(ifea3d *ctx)
{
    if (!ctx) return;
    delete ctx->s;
    delete ctx;
}

const char *ifea3d_last_error(const ifea3d *ctx) { return ctx && ctx->s ? ctx->s->err.c_str() : "null context"; }

ifea_status ifea3d_set_mesh(ifea3d *ctx, int32_t nn, int32_t ne, const double *x, const int32_t *tets,
                            const uint8_t *on_x0, const uint8_t *on_y0)
{
    if (!x || !tets || !on_x0 || !on_y0) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { s.set_mesh(nn, ne, x, tets, on_x0, on_y0); });
}

ifea_status ifea3d_set_die(ifea3d *ctx, int32_t side, int32_t nx, int32_t ny, double x0, double y0, double dx, const double *h)
{
    if (!h) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { s.set_die(side, nx, ny, x0, y0, dx, h); });
}

ifea_status ifea3d_set_trimesh_die(ifea3d *ctx, int32_t side, int32_t nv, const double *v, int32_t nt, const int32_t *tri)
{
    if (!v || !tri) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { s.set_trimesh_die(side, nv, v, nt, tri); });
}

ifea_status ifea3d_die_query(ifea3d *ctx, int32_t side, int32_t n, const double *p, double offset, double *clearance,
                             double *projected, double *normal, double *surface_z)
{
    if (n < 0 || (n > 0 && (!p || !clearance || !projected || !normal || !surface_z))) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { s.die_query(side, n, p, offset, clearance, projected, normal, surface_z); });
}

ifea_status ifea3d_init(ifea3d *ctx, double gap0, double min_x, double min_y, double min_z, double max_x, double max_y)
{
    return guarded(ctx, [&](Forging3D &s) { s.init(gap0, min_x, min_y, min_z, max_x, max_y); });
}

ifea_status ifea3d_step(ifea3d *ctx, ifea_step_info *info, const volatile int32_t *cancel)
{
    return guarded(ctx, [&](Forging3D &s) { s.step(info, cancel); });
}

ifea_status ifea3d_pattern_size(ifea3d *ctx, int64_t *nnz, int32_t *ndof)
{
    return guarded(ctx, [&](Forging3D &s) {
        if (nnz) *nnz = s.topo.nnz;
        if (ndof) *ndof = s.topo.ndof;
    });
}

ifea_status ifea3d_get_pattern(ifea3d *ctx, int32_t *col_ptr, int32_t *row_idx)
{
    return guarded(ctx, [&](Forging3D &s) {
        if (col_ptr) memcpy(col_ptr, s.topo.col_ptr.data(), s.topo.col_ptr.size() * sizeof(int32_t));
        if (row_idx) memcpy(row_idx, s.topo.row_idx.data(), s.topo.row_idx.size() * sizeof(int32_t));
    });
}

ifea_status ifea3d_prepare_step(ifea3d *ctx)
{
    return guarded(ctx, [&](Forging3D &s) { s.prepare_step(); });
}

ifea_status ifea3d_assemble(ifea3d *ctx, int32_t matrix, int32_t newton, const double *v_host, double *energy, double *power)
{
    return guarded(ctx, [&](Forging3D &s) {
        const double *v = s.d_vbuf[s.vcur];
        if (v_host) {
            s.d_vbuf[1 - s.vcur].upload(v_host, s.topo.ndof, s.st);
            v = s.d_vbuf[1 - s.vcur];
        }
        double e = s.assemble(matrix ? ifea::ASM_MATRIX : ifea::ASM_RESIDUAL, newton, v, false, power);
        if (energy) *energy = e;
    });
}

ifea_status ifea3d_apply_bc(ifea3d *ctx, double *max_diag)
{
    return guarded(ctx, [&](Forging3D &s) {
        s.apply_bc_separately();
        if (max_diag) *max_diag = s.max_diag;
    });
}

ifea_status ifea3d_solve_velocity(ifea3d *ctx, int32_t *iterations, int32_t *converged, const volatile int32_t *cancel)
{
    return guarded(ctx, [&](Forging3D &s) {
        bool conv = false;
        int it = s.solve_velocity(&conv, cancel);
        if (iterations) *iterations = it;
        if (converged) *converged = conv;
    });
}

ifea_status ifea3d_final_evaluation(ifea3d *ctx, double *power, double *reaction)
{
    return guarded(ctx, [&](Forging3D &s) {
        double p = s.final_evaluation(reaction);
        if (power) *power = p;
    });
}

ifea_status ifea3d_try_update(ifea3d *ctx, double dt, int32_t *ok)
{
    return guarded(ctx, [&](Forging3D &s) {
        std::string why;
        bool r = s.try_update(dt, why);
        if (ok) *ok = r;
        s.err = why;
    });
}

ifea_status ifea3d_set_stream(ifea3d *ctx, void *cuda_stream)
{
    return guarded(ctx, [&](Forging3D &s) { s.set_stream((cudaStream_t)cuda_stream); });
}

ifea_status ifea3d_time_factor_solve(ifea3d *ctx, double *ms)
{
    if (!ms) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { *ms = s.time_factor_solve(); });
}

ifea_status ifea3d_set_cavity(ifea3d *ctx, int32_t n, const double *xyz)
{
    return guarded(ctx, [&](Forging3D &s) { s.set_cavity(n, xyz); });
}

ifea_status ifea3d_fill_percent(ifea3d *ctx, double *pct)
{
    if (!pct) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { *pct = s.fill_percent(); });
}

const char *ifea3d_last_remesh(const ifea3d *ctx) { return ctx && ctx->s ? ctx->s->last_remesh.c_str() : ""; }

ifea_status ifea3d_set_warm_start(ifea3d *ctx, ifea_mlp *mlp, int32_t mode)
{
    if (mode < 0 || mode > 3 || (mode && (!mlp || !mlp->net))) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) {
        s.ws_net = mode ? mlp->net : nullptr;
        s.ws_mode = mode;
    });
}

ifea_status ifea3d_set_warm(ifea3d *ctx, int32_t warm)
{
    return guarded(ctx, [&](Forging3D &s) { s.warm = warm; });
}

ifea_status ifea3d_array_size(ifea3d *ctx, const char *name, int64_t *count, int32_t *elem_bytes)
{
    if (!name) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) {
        auto a = s.array(name);
        if (count) *count = (int64_t)a.count;
        if (elem_bytes) *elem_bytes = a.bytes < 0 ? -a.bytes : a.bytes;
    });
}

ifea_status ifea3d_get_array(ifea3d *ctx, const char *name, void *dst, int64_t count)
{
    if (!name || !dst) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) {
        auto a = s.array(name);
        if ((size_t)count != a.count) throw Failure(IFEA_INPUT_INVALID, "array size mismatch for '" + std::string(name) + "'");
        if (a.bytes < 0) {
            memcpy(dst, a.p, a.count * (size_t)(-a.bytes));
            return;
        }
        ifea::cuda_check(cudaMemcpyAsync(dst, a.p, a.count * (size_t)a.bytes, cudaMemcpyDeviceToHost, s.st), "D2H array");
        ifea::cuda_check(cudaStreamSynchronize(s.st), "cudaStreamSynchronize");
    });
}

ifea_status ifea3d_set_array(ifea3d *ctx, const char *name, const void *src, int64_t count)
{
    if (!name || !src) return IFEA_INPUT_INVALID;
    std::string nm(name);
    if (nm != "x" && nm != "vg" && nm != "eps" && nm != "el_sig" && nm != "contact" && nm != "v" && nm != "dmg" &&
        nm != "el_rate" && nm != "el_mean" && nm != "el_dev")
        return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) {
        auto a = s.array(nm);
        if ((size_t)count != a.count || a.bytes < 0) throw Failure(IFEA_INPUT_INVALID, "array size mismatch for '" + nm + "'");
        ifea::cuda_check(cudaMemcpyAsync(a.p, src, a.count * (size_t)a.bytes, cudaMemcpyHostToDevice, s.st), "H2D array");
        ifea::cuda_check(cudaStreamSynchronize(s.st), "cudaStreamSynchronize");
    });
}

ifea_status ifea3d_get_scalar(ifea3d *ctx, const char *name, double *value)
{
    if (!name || !value) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { *value = s.scalar(name); });
}

ifea_status ifea3d_set_scalar(ifea3d *ctx, const char *name, double value)
{
    if (!name) return IFEA_INPUT_INVALID;
    return guarded(ctx, [&](Forging3D &s) { s.set_scalar(name, value); });
}

}  // extern "C"
