// api.cu -- host implementation of the C ABI declared in include/rmhd2d.h.
//
// A solver owns two pitched SoA states (A: the current state U^n, B: the
// stage-1 state U*), an optional eta plane, the symmetric-wall row of CT'd
// bY, and a device control block (CFL maxima, dt, total time, crash and
// error flags).  One RK2 step is four launches on the solver's stream:
//
//   stage 1 (A -> B) ; boundary(B) ; stage 2 (B, A -> A) ; boundary(A) + CFL/NaN
//
// and the dt of step n+1 is reduced while step n finishes, so no host
// synchronisation happens inside a step (the reference synchronises on
// every boundary call and on the dt minimum, resistiveMHD_2D.cu:286-290).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rmhd2d.h"
#include "adjoint.h"
#include "aux_kernels.h"
#include "contact.h"
#include "noalloc_dt.h"
#include "physics.cuh"
#include "rmhd2d_internal.h"
#include "stage.cuh"

using namespace rmhd2d;

struct AdjointWork;

struct rmhd2d_solver {
    rmhd2d_config cfg{};
    Grid g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double *A = nullptr;         // current state, 8 planes
    double *B = nullptr;         // stage-1 state / staging, 8 planes
    double *eta = nullptr;       // eta plane or nullptr
    double *row2 = nullptr;      // nx doubles
    Control *ctl = nullptr;      // device control block
    Control *ctl_host = nullptr; // pinned mirror for readback
    // per tile shape: stage-1 source A, stage-2 source B, eta plane with the
    // stage-1 and stage-2 boxes
    CUtensorMap mapA[NSHAPE]{}, mapB[NSHAPE]{}, mapE1[NSHAPE]{}, mapE2[NSHAPE]{};
    int shape = 0;                       // tile shape of stage 1
    int shape2 = 0;                      // tile shape of stage 2
    void *batch = nullptr;               // owning batch, if any
    int parity = 0;
    bool has_state = false;
    long long steps = 0;
    cudaGraphExec_t graph2[2] = {nullptr, nullptr};
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};   // one step per parity (rmhd2d_step_rk2)
    AdjointWork *adj = nullptr;          // recorded trajectory and workspace of the discrete adjoint
    double *contact = nullptr;           // CT-Contact workspace: C, F1, G1, F2, G2 (8 planes each), R1, R2, E
    int slab = 0;                        // RMHD2D_SLAB_* flags of a slab of a decomposed domain (rmhd2d_create_slab)
    std::vector<float> tuning_ms;        // per tile shape: median ms of stage 1 and of stage 2 in the last autotune
    std::string err;
};

// Trajectory of rmhd2d_adjoint_forward and the workspace of
// rmhd2d_adjoint_backward (all device buffers are pitched like the state).
struct AdjointWork {
    int nsteps = 0, interval = 0, nseg = 0;
    int cap_steps = 0, cap_interval = 0, cap_seg = 0;   // sizes the buffers were allocated for
    bool tape = false;               // the forward run filled the segment slots with every step (no recompute)
    size_t state_doubles = 0;
    double *ckpt = nullptr;          // nseg states: U at steps 0, interval, 2*interval, ...
    double *seg0 = nullptr;          // interval states: U^n of each step of a segment (recomputed)
    double *seg1 = nullptr;          // interval states: U* of each step of a segment (recomputed)
    std::vector<CUtensorMap> map0, map1;   // stage-1 maps of the seg0 slots, stage-2 maps of the seg1 slots
    double *ub[3] = {nullptr, nullptr, nullptr};   // adjoint states
    double *Q = nullptr;             // 18 planes
    double *IF = nullptr;            // 32 planes
    double *RJ = nullptr;            // 6 planes
    double *tmp = nullptr;           // 2 planes
    double *etab = nullptr;          // 1 plane
    double *dts = nullptr;           // nsteps, device
    std::vector<double> dts_host;
    double *final_state = nullptr;   // U at the end of the forward run
    double *aos = nullptr;           // nx*ny*8 staging for seeds and gradients
    Control ctl_final{};
    bool recorded = false;           // the last forward run completed (nsteps, dts_host, final_state valid)
};

namespace {

std::mutex g_err_mu;
std::string g_create_err = "";

int fail(rmhd2d_solver *s, int code, const std::string &msg)
{
    if (s) {
        s->err = msg;
    } else {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_err = msg;
    }
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(s, RMHD2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
    } while (0)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 3-D tensor map over one state: (j: ny, i: nx, field: 8), box (uj, ui, 8).
bool encode_state_map(CUtensorMap *map, const Grid &g, double *base, int ui, int uj)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[3] = {(cuuint64_t)g.ny, (cuuint64_t)g.nx, (cuuint64_t)NFIELD};
    cuuint64_t strides[2] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.plane * 8};
    cuuint32_t box[3] = {(cuuint32_t)uj, (cuuint32_t)ui, (cuuint32_t)NFIELD};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 2-D tensor map over the eta plane: (j: ny, i: nx), box (uj, ui).
bool encode_eta_map(CUtensorMap *map, const Grid &g, double *base, int ui, int uj)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)g.ny, (cuuint64_t)g.nx};
    cuuint64_t strides[1] = {(cuuint64_t)g.pitch * 8};
    cuuint32_t box[2] = {(cuuint32_t)uj, (cuuint32_t)ui};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

int sync_and_check(rmhd2d_solver *s)
{
    // The control block is read behind the stream's work: one wait covers both.
    CK(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Control), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    if (s->ctl_host->error != KERR_NONE)
        return fail(s, RMHD2D_ERR_KERNEL, "a stage kernel's bounded wait for its staged tile expired");
    return RMHD2D_OK;
}

// Re-reduces the CFL rate and crash flag of the current state into slot
// `parity` (after a state change outside a step).
int refresh_rate(rmhd2d_solver *s)
{
    CK(cudaMemsetAsync(&s->ctl->amax[s->parity], 0, sizeof(unsigned long long), s->stream));
    CK(cudaMemsetAsync(&s->ctl->first_nan[s->parity], 0, sizeof(int), s->stream));
    CK(cudaMemsetAsync(&s->ctl->crashed, 0, sizeof(int), s->stream));
    launch_rate(s->g, s->A, s->ctl, s->parity, 1, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int do_boundary(rmhd2d_solver *s)
{
    if (s->g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(s->g, s->A, s->row2, s->stream);
    launch_boundary(s->g, s->A, s->row2, nullptr, 0, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

// rmhd2d_solver::slab: set (with the RMHD2D_SLAB_* flags) by rmhd2d_create_slab.
constexpr int SLAB_CREATED = 1 << 8;

// Entry points that step, fill or reduce over the whole array refuse a slab
// with halo columns: its neighbours' exchange and the cross-slab reduction
// are steps the host takes between the rmhd2d_slab_* calls.
int refuse_halo_slab(rmhd2d_solver *s, const char *what)
{
    return fail(s, RMHD2D_ERR_STATE,
                std::string(what) + " on a slab with halo columns: step it with rmhd2d_slab_stage / "
                                    "rmhd2d_slab_fill and the host's exchange");
}

using StageLauncher = void (*)(int, int, const CUtensorMap *, const CUtensorMap *, const StageArgs &, cudaStream_t);
using BatchLauncher = void (*)(int, int, const BatchRun *, const CUtensorMap *, const TileRef *, int, int, int,
                               cudaStream_t);

StageLauncher stage_launcher(int precision)
{
    switch (precision) {
    case RMHD2D_FP64_FAST: return fast::launch_stage;
    case RMHD2D_FP32_BULK: return bulk32::launch_stage;
    default: return exact::launch_stage;
    }
}

BatchLauncher batch_launcher(int precision)
{
    switch (precision) {
    case RMHD2D_FP64_FAST: return fast::launch_stage_batch;
    case RMHD2D_FP32_BULK: return bulk32::launch_stage_batch;
    default: return exact::launch_stage_batch;
    }
}

// One stage-1-EMF step from `un` (read through map_un) into `dst`, with U*
// in `ustar` (read through map_ustar); the same launches as enqueue_step
// without A and B.  dst may not be un.
void enqueue_step_between(rmhd2d_solver *s, int parity, const double *un, const CUtensorMap *map_un, double *ustar,
                          const CUtensorMap *map_ustar, double *dst, double *dt_log, const double *dt_in)
{
    StageArgs a{};
    a.dt_in = dt_in;
    a.g = s->g;
    a.eta = s->eta;
    a.row2 = s->g.bc_x == BC_SYMMETRIC ? s->row2 : nullptr;
    a.ctl = s->ctl;
    a.parity = parity;
    auto launch = stage_launcher(s->cfg.precision);
    a.src = un;
    a.un = un;
    a.dst = ustar;
    a.dt_log = dt_log;
    launch(1, s->shape, map_un, &s->mapE1[s->shape], a, s->stream);
    a.dt_log = nullptr;
    launch_boundary(s->g, ustar, s->row2, nullptr, 0, s->stream);
    a.src = ustar;
    a.un = un;
    a.dst = dst;
    launch(2, s->shape2, map_ustar, &s->mapE2[s->shape2], a, s->stream);
    launch_boundary(s->g, dst, s->row2, s->ctl, parity ^ 1, s->stream);
}

// dt_log: stage 1 also writes the step's dt there (a recorded run); dt_in:
// the step reads its dt from there (a replayed run).  Not for CT-Contact,
// whose pipeline takes its dt from the control block.
void enqueue_step(rmhd2d_solver *s, int parity, double *dt_log = nullptr, const double *dt_in = nullptr)
{
    if (s->contact) {
        const size_t P = (size_t)s->g.plane;
        ContactStep c{};
        c.g = s->g;
        c.A = s->A;
        c.B = s->B;
        c.C = s->contact;
        c.F1 = c.C + NFIELD * P;
        c.G1 = c.F1 + NFIELD * P;
        c.F2 = c.G1 + NFIELD * P;
        c.G2 = c.F2 + NFIELD * P;
        c.R1 = c.G2 + NFIELD * P;
        c.R2 = c.R1 + P;
        c.E = c.R2 + P;
        c.eta = s->eta;
        c.row2 = s->row2;
        c.ctl = s->ctl;
        c.parity = parity;
        enqueue_contact_step(c, s->stream);
        return;
    }
    StageArgs a{};
    a.g = s->g;
    a.eta = s->eta;
    a.row2 = s->g.bc_x == BC_SYMMETRIC ? s->row2 : nullptr;
    a.ctl = s->ctl;
    a.parity = parity;
    a.dt_in = dt_in;
    auto launch = stage_launcher(s->cfg.precision);
    // stage 1: U^n (A) -> U* (B)
    a.src = s->A;
    a.un = s->A;
    a.dst = s->B;
    a.dt_log = dt_log;
    launch(1, s->shape, &s->mapA[s->shape], &s->mapE1[s->shape], a, s->stream);
    a.dt_log = nullptr;
    launch_boundary(s->g, s->B, s->row2, nullptr, 0, s->stream);
    // stage 2: (U*, U^n) -> U^{n+1} in A
    a.src = s->B;
    a.un = s->A;
    a.dst = s->A;
    launch(2, s->shape2, &s->mapB[s->shape2], &s->mapE2[s->shape2], a, s->stream);
    launch_boundary(s->g, s->A, s->row2, s->ctl, parity ^ 1, s->stream);
}

int upload_from_device_aos(rmhd2d_solver *s, const double *aos_dev, int apply_boundary)
{
    launch_aos_to_planes(s->g, aos_dev, s->A, s->stream);
    CK(cudaGetLastError());
    s->has_state = true;
    if (apply_boundary) {
        int rc = do_boundary(s);
        if (rc) return rc;
    }
    return refresh_rate(s);
}

void free_adjoint(AdjointWork *w)
{
    if (!w) return;
    cudaFree(w->ckpt);
    cudaFree(w->seg0);
    cudaFree(w->seg1);
    for (double *p : w->ub) cudaFree(p);
    cudaFree(w->Q);
    cudaFree(w->IF);
    cudaFree(w->RJ);
    cudaFree(w->tmp);
    cudaFree(w->etab);
    cudaFree(w->dts);
    cudaFree(w->final_state);
    cudaFree(w->aos);
    delete w;
}

// Sets or clears Control::use_fixed_dt in stream order.
int set_fixed_dt_mode(rmhd2d_solver *s, int on)
{
    static const int kOn = 1, kOff = 0;
    CK(cudaMemcpyAsync(&s->ctl->use_fixed_dt, on ? &kOn : &kOff, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    return RMHD2D_OK;
}

// A device buffer freed on scope exit.
struct DeviceBuffer {
    double *p = nullptr;
    ~DeviceBuffer() { cudaFree(p); }
};

// A CUDA event destroyed on scope exit.
struct ScopedEvent {
    cudaEvent_t e = nullptr;
    ScopedEvent() = default;
    ScopedEvent(const ScopedEvent &) = delete;
    ScopedEvent &operator=(const ScopedEvent &) = delete;
    ~ScopedEvent()
    {
        if (e) cudaEventDestroy(e);
    }
};

// Turns Control::use_fixed_dt back off when a frozen-dt run returns early, so
// that later steps take the CFL dt again.  The error already reported is kept.
struct FixedDtScope {
    rmhd2d_solver *s = nullptr;
    bool armed = false;
    ~FixedDtScope()
    {
        static const int kOff = 0;
        if (armed)
            cudaMemcpyAsync(&s->ctl->use_fixed_dt, &kOff, sizeof(int), cudaMemcpyHostToDevice, s->stream);
    }
};

void destroy_graphs(rmhd2d_solver *s)
{
    for (auto &gx : s->graph2) {
        if (gx) cudaGraphExecDestroy(gx);
        gx = nullptr;
    }
    for (auto &gx : s->graph1) {
        if (gx) cudaGraphExecDestroy(gx);
        gx = nullptr;
    }
}

}  // namespace

extern "C" {

void rmhd2d_config_default(rmhd2d_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->nx = c->ny = 0;
    c->dx = c->dy = 1.0;
    c->gamma_mhd = 5.0 / 3.0;
    c->cfl = 0.4;
    c->eps = 1e-20;
    c->eta = 0.0;
    c->bc = RMHD2D_BC_PERIODIC;
    c->bc_y = -1;
    c->precision = RMHD2D_FP64_EXACT;
    c->device = 0;
    c->stream = nullptr;
    c->ct_scheme = RMHD2D_CT_STAGE1;
}

int rmhd2d_abi_version(void) { return RMHD2D_ABI_VERSION; }

const char *rmhd2d_status_string(int st)
{
    switch (st) {
    case RMHD2D_OK: return "ok";
    case RMHD2D_ERR_INVALID: return "invalid argument";
    case RMHD2D_ERR_CUDA: return "CUDA error";
    case RMHD2D_ERR_NO_DEVICE: return "no sm_100 device";
    case RMHD2D_ERR_STATE: return "invalid solver state";
    case RMHD2D_ERR_IO: return "I/O error";
    case RMHD2D_ERR_KERNEL: return "kernel error";
    default: return "unknown status";
    }
}

const char *rmhd2d_last_error(const rmhd2d_solver *s)
{
    if (s) return s->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_create_err.c_str();
}

int rmhd2d_create(const rmhd2d_config *cfg, rmhd2d_solver **out)
{
    rmhd2d_solver *s = nullptr;
    if (!cfg || !out) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->nx < 12 || cfg->ny < 12) return fail(s, RMHD2D_ERR_INVALID, "nx and ny must be >= 12 (3 ghosts per side)");
    if ((long long)cfg->nx * cfg->ny > (1LL << 31)) return fail(s, RMHD2D_ERR_INVALID, "grid too large");
    if (!(cfg->dx > 0) || !(cfg->dy > 0)) return fail(s, RMHD2D_ERR_INVALID, "dx and dy must be positive");
    if (!(cfg->gamma_mhd > 1.0)) return fail(s, RMHD2D_ERR_INVALID, "gamma_mhd must be > 1");
    if (!(cfg->eta >= 0.0)) return fail(s, RMHD2D_ERR_INVALID, "eta must be >= 0");
    {
        const int bx = cfg->bc, by = cfg->bc_y == -1 ? cfg->bc : cfg->bc_y;
        if (bx != RMHD2D_BC_PERIODIC && bx != RMHD2D_BC_SYMMETRIC && bx != RMHD2D_BC_ZERO_GRADIENT &&
            bx != RMHD2D_BC_FLARE)
            return fail(s, RMHD2D_ERR_INVALID, "unknown x boundary kind (wall walls are y walls)");
        if (by != RMHD2D_BC_PERIODIC && by != RMHD2D_BC_SYMMETRIC && by != RMHD2D_BC_ZERO_GRADIENT &&
            by != RMHD2D_BC_WALL)
            return fail(s, RMHD2D_ERR_INVALID, "unknown y boundary kind (flare walls are x walls; set bc_y)");
    }
    if (cfg->precision != RMHD2D_FP64_EXACT && cfg->precision != RMHD2D_FP64_FAST &&
        cfg->precision != RMHD2D_FP32_BULK)
        return fail(s, RMHD2D_ERR_INVALID, "unknown precision");
    if (cfg->ct_scheme != RMHD2D_CT_STAGE1 && cfg->ct_scheme != RMHD2D_CT_CONTACT)
        return fail(s, RMHD2D_ERR_INVALID, "unknown ct_scheme");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0)
        return fail(s, RMHD2D_ERR_NO_DEVICE, "no CUDA device with that ordinal");
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10 || prop.minor != 0)
        return fail(s, RMHD2D_ERR_NO_DEVICE, "librmhd2d is built for sm_100a (B200) only");

    s = new rmhd2d_solver();
    s->cfg = *cfg;
    s->device = cfg->device;
    Grid &g = s->g;
    g.nx = cfg->nx;
    g.ny = cfg->ny;
    g.pitch = (cfg->ny + 31) / 32 * 32;
    g.plane = (long long)g.nx * g.pitch;
    g.dx = cfg->dx;
    g.dy = cfg->dy;
    g.gamma = cfg->gamma_mhd;
    g.cfl = cfg->cfl;
    g.eps = cfg->eps;
    g.eta = cfg->eta;
    g.bc_x = cfg->bc;
    g.bc_y = cfg->bc_y < 0 ? cfg->bc : cfg->bc_y;

    auto bail = [&](int code, const std::string &msg) {
        {
            std::lock_guard<std::mutex> lk(g_err_mu);
            g_create_err = msg;
        }
        rmhd2d_destroy(s);
        return code;
    };
    if (cudaSetDevice(s->device) != cudaSuccess) return bail(RMHD2D_ERR_CUDA, "cudaSetDevice failed");
    if (cfg->stream) {
        s->stream = (cudaStream_t)cfg->stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(RMHD2D_ERR_CUDA, "cudaStreamCreate failed");
        s->own_stream = true;
    }
    const size_t state_bytes = (size_t)g.plane * NFIELD * sizeof(double);
    if (cudaMalloc(&s->A, state_bytes) != cudaSuccess || cudaMalloc(&s->B, state_bytes) != cudaSuccess ||
        cudaMalloc(&s->row2, (size_t)g.nx * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&s->ctl, sizeof(Control)) != cudaSuccess ||
        cudaMallocHost(&s->ctl_host, sizeof(Control)) != cudaSuccess)
        return bail(RMHD2D_ERR_CUDA, "device allocation failed");
    // Every clear goes on the solver's stream, which does not synchronise
    // with the legacy default stream (cudaStreamNonBlocking): a plain
    // cudaMemset there could still be running when set_state's copy lands
    // and zero part of it.  The stream is drained before create returns.
    if (cfg->ct_scheme == RMHD2D_CT_CONTACT) {
        const size_t cbytes = (size_t)g.plane * (5 * NFIELD + 3) * sizeof(double);
        if (cudaMalloc(&s->contact, cbytes) != cudaSuccess ||
            cudaMemsetAsync(s->contact, 0, cbytes, s->stream) != cudaSuccess)
            return bail(RMHD2D_ERR_CUDA, "device allocation failed (CT-Contact workspace)");
    }
    // Zero the planes so padding columns hold finite values.
    if (cudaMemsetAsync(s->A, 0, state_bytes, s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->B, 0, state_bytes, s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->row2, 0, (size_t)g.nx * sizeof(double), s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->ctl, 0, sizeof(Control), s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess)
        return bail(RMHD2D_ERR_CUDA, "device memset failed");
    for (int sh = 0; sh < NSHAPE; ++sh)
        if (!encode_state_map(&s->mapA[sh], g, s->A, stage_ui(1, sh), shape_uj(sh)) ||
            !encode_state_map(&s->mapB[sh], g, s->B, stage_ui(2, sh), shape_uj(sh)))
            return bail(RMHD2D_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    *out = s;
    return RMHD2D_OK;
}

static int destroy_solver(rmhd2d_solver *s);

int rmhd2d_destroy(rmhd2d_solver *s)
{
    if (!s) return RMHD2D_OK;
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: destroy the batch");
    return destroy_solver(s);
}

static int destroy_solver(rmhd2d_solver *s)
{
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    destroy_graphs(s);
    cudaFree(s->A);
    cudaFree(s->B);
    cudaFree(s->eta);
    cudaFree(s->row2);
    cudaFree(s->ctl);
    cudaFree(s->contact);
    free_adjoint(s->adj);
    if (s->ctl_host) cudaFreeHost(s->ctl_host);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return RMHD2D_OK;
}

int rmhd2d_set_state(rmhd2d_solver *s, const double *host, int apply_boundary)
{
    if (!s || !host) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (apply_boundary && s->g.x_halo) return refuse_halo_slab(s, "set_state with apply_boundary");
    CK(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.nx * s->g.ny * NFIELD;
    // B doubles as the AoS staging buffer (it holds no live data between steps).
    CK(cudaMemcpyAsync(s->B, host, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    return upload_from_device_aos(s, s->B, apply_boundary);
}

int rmhd2d_set_state_device(rmhd2d_solver *s, const double *dev, int apply_boundary)
{
    if (!s || !dev) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (apply_boundary && s->g.x_halo) return refuse_halo_slab(s, "set_state_device with apply_boundary");
    CK(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.nx * s->g.ny * NFIELD;
    CK(cudaMemcpyAsync(s->B, dev, n * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    return upload_from_device_aos(s, s->B, apply_boundary);
}

int rmhd2d_get_state(rmhd2d_solver *s, double *host)
{
    if (!s || !host) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    const size_t n = (size_t)s->g.nx * s->g.ny * NFIELD;
    launch_planes_to_aos(s->g, s->A, s->B, s->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, s->B, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    return sync_and_check(s);
}

int rmhd2d_set_eta_table(rmhd2d_solver *s, const double *host_eta)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    destroy_graphs(s);
    if (!host_eta) {
        cudaFree(s->eta);
        s->eta = nullptr;
        return RMHD2D_OK;
    }
    if (!s->eta) {
        CK(cudaMalloc(&s->eta, (size_t)s->g.plane * sizeof(double)));
        CK(cudaMemsetAsync(s->eta, 0, (size_t)s->g.plane * sizeof(double), s->stream));
        bool ok = true;
        for (int sh = 0; sh < NSHAPE; ++sh)
            ok = ok && encode_eta_map(&s->mapE1[sh], s->g, s->eta, stage_ui(1, sh), shape_uj(sh)) &&
                 encode_eta_map(&s->mapE2[sh], s->g, s->eta, stage_ui(2, sh), shape_uj(sh));
        if (!ok) {
            cudaFree(s->eta);
            s->eta = nullptr;
            return fail(s, RMHD2D_ERR_CUDA, "cuTensorMapEncodeTiled failed for the eta table");
        }
    }
    CK(cudaMemcpy2DAsync(s->eta, (size_t)s->g.pitch * sizeof(double), host_eta, (size_t)s->g.ny * sizeof(double),
                         (size_t)s->g.ny * sizeof(double), (size_t)s->g.nx, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return RMHD2D_OK;
}

int rmhd2d_apply_boundary(rmhd2d_solver *s)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "apply_boundary");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    int rc = do_boundary(s);
    if (rc) return rc;
    return refresh_rate(s);
}

int rmhd2d_calculate_dt(rmhd2d_solver *s, double *dt)
{
    if (!s || !dt) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (s->g.x_halo) return refuse_halo_slab(s, "calculate_dt");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    int rc = sync_and_check(s);
    if (rc) return rc;
    const Grid &g = s->g;
    *dt = step_dt(s->ctl_host->amax[s->parity], s->ctl_host->first_nan[s->parity], g.dx, g.dy, g.eps, g.eta, g.cfl);
    return RMHD2D_OK;
}

// Captures `nsteps` consecutive steps starting at step parity `parity` into
// *ge and uploads the graph, so that its first launch costs no more than
// the later ones.
static int capture_steps(rmhd2d_solver *s, int parity, int nsteps, cudaGraphExec_t *ge)
{
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (int n = 0; n < nsteps; ++n) enqueue_step(s, parity ^ (n & 1));
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (e != cudaSuccess) return fail(s, RMHD2D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(ge, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        *ge = nullptr;
        return fail(s, RMHD2D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    CK(cudaGraphUpload(*ge, s->stream));
    return RMHD2D_OK;
}

// The one-step (k = 1) or two-step (k = 2) graphs of both step parities,
// captured together on first use: a run's step count then never meets an
// uncaptured parity, so no capture falls inside a later (timed) run.
static int ensure_step_graphs(rmhd2d_solver *s, cudaGraphExec_t g[2], int k)
{
    for (int p = 0; p < 2; ++p)
        if (!g[p]) {
            const int rc = capture_steps(s, p, k, &g[p]);
            if (rc) return rc;
        }
    return RMHD2D_OK;
}

int rmhd2d_step_rk2(rmhd2d_solver *s)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "step_rk2");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: step the batch");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    // One step replayed from a captured graph: a single launch instead of
    // the step's kernels one by one, which is what a driver loop that
    // synchronises after every step (crash check, dt) waits on.  Under a
    // caller's own stream capture the kernels are enqueued directly.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        enqueue_step(s, s->parity);
        CK(cudaGetLastError());
    } else {
        const int rc = ensure_step_graphs(s, s->graph1, 1);
        if (rc) return rc;
        CK(cudaGraphLaunch(s->graph1[s->parity], s->stream));
    }
    s->parity ^= 1;
    s->steps += 1;
    return RMHD2D_OK;
}

int rmhd2d_run(rmhd2d_solver *s, int nsteps)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "run");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: step the batch");
    if (nsteps < 0) return fail(s, RMHD2D_ERR_INVALID, "nsteps < 0");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    if (nsteps >= 2) {
        const int rc = ensure_step_graphs(s, s->graph2, 2);
        if (rc) return rc;
    }
    while (nsteps >= 2) {
        CK(cudaGraphLaunch(s->graph2[s->parity], s->stream));
        s->steps += 2;
        nsteps -= 2;
    }
    if (nsteps == 1) return rmhd2d_step_rk2(s);
    return RMHD2D_OK;
}

int rmhd2d_run_timed(rmhd2d_solver *s, int nsteps, float *ms)
{
    if (!s || !ms) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    ScopedEvent e0, e1;
    CK(cudaEventCreate(&e0.e));
    CK(cudaEventCreate(&e1.e));
    CK(cudaEventRecord(e0.e, s->stream));
    int rc = rmhd2d_run(s, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(e1.e, s->stream));
    CK(cudaEventSynchronize(e1.e));
    CK(cudaEventElapsedTime(ms, e0.e, e1.e));
    return sync_and_check(s);
}

int rmhd2d_profile_step(rmhd2d_solver *s, float *ms4)
{
    if (!s || !ms4) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (s->g.x_halo) return refuse_halo_slab(s, "profile_step");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: step the batch");
    if (s->contact) return fail(s, RMHD2D_ERR_STATE, "profile_step times the four launches of the stage-1-EMF step");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    ScopedEvent sev[5];
    cudaEvent_t ev[5];
    for (int n = 0; n < 5; ++n) {
        CK(cudaEventCreate(&sev[n].e));
        ev[n] = sev[n].e;
    }
    const int parity = s->parity;
    StageArgs a{};
    a.g = s->g;
    a.eta = s->eta;
    a.row2 = s->g.bc_x == BC_SYMMETRIC ? s->row2 : nullptr;
    a.ctl = s->ctl;
    a.parity = parity;
    auto launch = stage_launcher(s->cfg.precision);
    CK(cudaEventRecord(ev[0], s->stream));
    a.src = s->A; a.un = s->A; a.dst = s->B;
    launch(1, s->shape, &s->mapA[s->shape], &s->mapE1[s->shape], a, s->stream);
    CK(cudaEventRecord(ev[1], s->stream));
    launch_boundary(s->g, s->B, s->row2, nullptr, 0, s->stream);
    CK(cudaEventRecord(ev[2], s->stream));
    a.src = s->B; a.un = s->A; a.dst = s->A;
    launch(2, s->shape2, &s->mapB[s->shape2], &s->mapE2[s->shape2], a, s->stream);
    CK(cudaEventRecord(ev[3], s->stream));
    launch_boundary(s->g, s->A, s->row2, s->ctl, parity ^ 1, s->stream);
    CK(cudaEventRecord(ev[4], s->stream));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev[4]));
    for (int n = 0; n < 4; ++n) CK(cudaEventElapsedTime(&ms4[n], ev[n], ev[n + 1]));
    s->parity ^= 1;
    s->steps += 1;
    return sync_and_check(s);
}

int rmhd2d_get_dt(rmhd2d_solver *s, double *dt)
{
    if (!s || !dt) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    int rc = sync_and_check(s);
    if (rc) return rc;
    *dt = s->ctl_host->dt;
    return RMHD2D_OK;
}

int rmhd2d_get_total_time(rmhd2d_solver *s, double *t)
{
    if (!s || !t) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    int rc = sync_and_check(s);
    if (rc) return rc;
    *t = s->ctl_host->total_time;
    return RMHD2D_OK;
}

int rmhd2d_check_crashed(rmhd2d_solver *s, int *crashed)
{
    if (!s || !crashed) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    int rc = sync_and_check(s);
    if (rc) return rc;
    *crashed = s->ctl_host->crashed ? 1 : 0;
    return RMHD2D_OK;
}

int rmhd2d_write_snapshot(const char *path, const double *host_state, int nx, int ny)
{
    rmhd2d_solver *s = nullptr;
    if (!path || !host_state || nx <= 0 || ny <= 0) return fail(s, RMHD2D_ERR_INVALID, "bad snapshot arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(s, RMHD2D_ERR_IO, std::string("cannot open ") + path);
    // The reference's save() loops (resistiveMHD_2D.cu:214-243) emit every
    // cell k = 0 .. nx*ny-1 in order, 8 raw doubles each.
    const size_t n = (size_t)nx * ny * NFIELD;
    const size_t w = std::fwrite(host_state, sizeof(double), n, f);
    const int closed = std::fclose(f);
    if (w != n || closed != 0) return fail(s, RMHD2D_ERR_IO, std::string("short write to ") + path);
    return RMHD2D_OK;
}

int rmhd2d_save(rmhd2d_solver *s, const char *dir, const char *name, int step)
{
    if (!s || !dir || !name) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    std::vector<double> h((size_t)s->g.nx * s->g.ny * NFIELD);
    int rc = rmhd2d_get_state(s, h.data());
    if (rc) return rc;
    const std::string path = std::string(dir) + "/" + name + "_" + std::to_string(step) + ".bin";
    rc = rmhd2d_write_snapshot(path.c_str(), h.data(), s->g.nx, s->g.ny);
    if (rc) return fail(s, rc, std::string("cannot write ") + path);
    return RMHD2D_OK;
}

int rmhd2d_load(rmhd2d_solver *s, const char *path)
{
    if (!s || !path) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    const size_t n = (size_t)s->g.nx * s->g.ny * NFIELD;
    std::vector<double> h(n);
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(s, RMHD2D_ERR_IO, std::string("cannot open ") + path);
    const size_t r = std::fread(h.data(), sizeof(double), n, f);
    const int extra = std::fgetc(f);
    std::fclose(f);
    if (r != n || extra != EOF) return fail(s, RMHD2D_ERR_IO, std::string("size mismatch reading ") + path);
    int rc = rmhd2d_set_state(s, h.data(), 0);
    if (rc) return rc;
    return sync_and_check(s);
}


// ---------------------------------------------------------------------------
// Tile shape and autotuning of one solver
// ---------------------------------------------------------------------------

int rmhd2d_set_stage_shapes(rmhd2d_solver *s, int shape1, int shape2)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (shape1 < 0 || shape1 >= NSHAPE || shape2 < 0 || shape2 >= NSHAPE)
        return fail(s, RMHD2D_ERR_INVALID, "unknown tile shape");
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    destroy_graphs(s);
    s->shape = shape1;
    s->shape2 = shape2;
    return RMHD2D_OK;
}

int rmhd2d_get_stage_shapes(const rmhd2d_solver *s, int *shape1, int *shape2)
{
    if (!s || !shape1 || !shape2) return fail(const_cast<rmhd2d_solver *>(s), RMHD2D_ERR_INVALID, "null argument");
    *shape1 = s->shape;
    *shape2 = s->shape2;
    return RMHD2D_OK;
}

int rmhd2d_set_tile_shape(rmhd2d_solver *s, int shape) { return rmhd2d_set_stage_shapes(s, shape, shape); }

int rmhd2d_get_tuning(const rmhd2d_solver *s, int max, int *n, int *shapes, float *ms_stage1, float *ms_stage2)
{
    if (!s || !n) return fail(const_cast<rmhd2d_solver *>(s), RMHD2D_ERR_INVALID, "null argument");
    const int k = (int)s->tuning_ms.size() / 2;
    *n = k;
    for (int q = 0; q < k && q < max; ++q) {
        if (shapes) shapes[q] = q;
        if (ms_stage1) ms_stage1[q] = s->tuning_ms[2 * q];
        if (ms_stage2) ms_stage2[q] = s->tuning_ms[2 * q + 1];
    }
    return RMHD2D_OK;
}

int rmhd2d_get_tile_shape(const rmhd2d_solver *s, int *shape)
{
    if (!s || !shape) return RMHD2D_ERR_INVALID;
    *shape = s->shape;
    return RMHD2D_OK;
}

// Saves the user-visible state (A and the control block) of a solver so that
// trial steps can be undone.
struct Snapshot {
    double *A = nullptr;   // owned: freed on restore or on scope exit
    Control ctl{};
    int parity = 0;
    long long steps = 0;
    Snapshot() = default;
    Snapshot(const Snapshot &) = delete;
    Snapshot &operator=(const Snapshot &) = delete;
    ~Snapshot() { cudaFree(A); }
};

static int snapshot_take(rmhd2d_solver *s, Snapshot &sn)
{
    const size_t bytes = (size_t)s->g.plane * NFIELD * sizeof(double);
    CK(cudaMalloc(&sn.A, bytes));
    CK(cudaMemcpyAsync(sn.A, s->A, bytes, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(&sn.ctl, s->ctl, sizeof(Control), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    sn.parity = s->parity;
    sn.steps = s->steps;
    return RMHD2D_OK;
}

static int snapshot_restore(rmhd2d_solver *s, Snapshot &sn)
{
    const size_t bytes = (size_t)s->g.plane * NFIELD * sizeof(double);
    CK(cudaMemcpyAsync(s->A, sn.A, bytes, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->ctl, &sn.ctl, sizeof(Control), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(sn.A);
    sn.A = nullptr;
    s->parity = sn.parity;
    s->steps = sn.steps;
    return RMHD2D_OK;
}

int rmhd2d_autotune(rmhd2d_solver *s, int trial_steps, int *best_shape)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "autotune");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: tune the batch");
    if (s->contact) {   // the CT-Contact pipeline does not run the tiled stage kernels
        if (best_shape) *best_shape = s->shape;
        return RMHD2D_OK;
    }
    if (trial_steps < 2) trial_steps = 2;
    trial_steps += trial_steps & 1;   // even: the step parity comes back
    CK(cudaSetDevice(s->device));
    Snapshot sn;
    int rc = snapshot_take(s, sn);
    if (rc) return rc;
    // Each stage's launch is timed by itself (the two stages read and write
    // different tiles and buffers), so the fastest shape is picked per stage:
    // the median over trial steps of each stage's CUDA-event time.
    s->tuning_ms.assign(2 * NSHAPE, 0.f);
    for (int sh = 0; sh < NSHAPE && rc == RMHD2D_OK; ++sh) {
        rc = rmhd2d_set_stage_shapes(s, sh, sh);
        if (!rc) rc = rmhd2d_run(s, 2);                          // warm-up
        std::vector<float> t1, t2;
        for (int k = 0; k < trial_steps && !rc; ++k) {
            float ms4[4];
            rc = rmhd2d_profile_step(s, ms4);
            t1.push_back(ms4[0]);
            t2.push_back(ms4[2]);
        }
        if (!rc) {
            std::sort(t1.begin(), t1.end());
            std::sort(t2.begin(), t2.end());
            s->tuning_ms[2 * sh] = t1[t1.size() / 2];
            s->tuning_ms[2 * sh + 1] = t2[t2.size() / 2];
        }
    }
    const int rc2 = snapshot_restore(s, sn);
    if (rc) return rc;
    if (rc2) return rc2;
    int b1 = 0, b2 = 0;
    for (int sh = 1; sh < NSHAPE; ++sh) {
        if (s->tuning_ms[2 * sh] < s->tuning_ms[2 * b1]) b1 = sh;
        if (s->tuning_ms[2 * sh + 1] < s->tuning_ms[2 * b2 + 1]) b2 = sh;
    }
    rc = rmhd2d_set_stage_shapes(s, b1, b2);
    if (best_shape) *best_shape = b1;
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches of independent runs
// ---------------------------------------------------------------------------

struct rmhd2d_batch {
    std::vector<rmhd2d_solver *> runs;
    int device = 0;
    int precision = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nsm = 148;
    int shape = 0;
    int ctas_per_sm = 2;
    int parity = 0;
    long long steps = 0;
    long long max_ghost = 0;
    BatchRun *d_runs = nullptr;
    CUtensorMap *d_maps = nullptr;            // MAPS_PER_RUN per run, for the current shape
    TileRef *d_tiles[2] = {nullptr, nullptr}; // stage 1 / stage 2 tile tables
    int ntiles[2] = {0, 0};
    bool dirty = true;
    cudaGraphExec_t graph2[2] = {nullptr, nullptr};
    // (tile shape, CTAs per SM, ms per step) of each point of the last rmhd2d_batch_autotune
    std::vector<int> tune_shape, tune_ctas;
    std::vector<float> tune_ms;
    std::string err;
};

namespace {

int bfail(rmhd2d_batch *b, int code, const std::string &msg)
{
    if (b) b->err = msg;
    else {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_create_err = msg;
    }
    return code;
}

#define BCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return bfail(b, RMHD2D_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void batch_drop_graphs(rmhd2d_batch *b)
{
    for (auto &g : b->graph2) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// (Re)builds the device run records, tensor maps and tile tables.
int batch_build(rmhd2d_batch *b)
{
    if (!b->dirty) return RMHD2D_OK;
    BCK(cudaStreamSynchronize(b->stream));
    batch_drop_graphs(b);
    const int n = (int)b->runs.size();
    std::vector<BatchRun> runs(n);
    std::vector<CUtensorMap> maps((size_t)n * MAPS_PER_RUN);
    std::vector<TileRef> tiles[2];
    b->max_ghost = 0;
    for (int r = 0; r < n; ++r) {
        rmhd2d_solver *s = b->runs[r];
        if (!s->has_state) return bfail(b, RMHD2D_ERR_STATE, "run " + std::to_string(r) + " has no state");
        runs[r] = BatchRun{s->g, s->A, s->B, s->eta, s->row2, s->ctl};
        maps[(size_t)r * MAPS_PER_RUN + 0] = s->mapA[b->shape];
        maps[(size_t)r * MAPS_PER_RUN + 1] = s->mapB[b->shape];
        maps[(size_t)r * MAPS_PER_RUN + 2] = s->mapE1[b->shape];
        maps[(size_t)r * MAPS_PER_RUN + 3] = s->mapE2[b->shape];
        const long long ng = 6LL * s->g.ny + 6LL * (s->g.nx - 6);
        b->max_ghost = ng > b->max_ghost ? ng : b->max_ghost;
        for (int st = 1; st <= 2; ++st) {
            const int ti = stage_ti(st, b->shape), tj = shape_tj(b->shape);
            const int nti = (s->g.nx - 2 * HALO + ti - 1) / ti, ntj = (s->g.ny - 2 * HALO + tj - 1) / tj;
            for (int a = 0; a < nti; ++a)
                for (int c = 0; c < ntj; ++c) tiles[st - 1].push_back(TileRef{r, a, c, 0});
        }
    }
    cudaFree(b->d_runs);
    cudaFree(b->d_maps);
    b->d_runs = nullptr;
    b->d_maps = nullptr;
    BCK(cudaMalloc(&b->d_runs, sizeof(BatchRun) * n));
    BCK(cudaMalloc(&b->d_maps, sizeof(CUtensorMap) * maps.size()));
    // On the batch stream (not the legacy default stream, which the batch
    // stream does not wait for), drained before the host tables go away.
    BCK(cudaMemcpyAsync(b->d_runs, runs.data(), sizeof(BatchRun) * n, cudaMemcpyHostToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                        b->stream));
    for (int st = 0; st < 2; ++st) {
        cudaFree(b->d_tiles[st]);
        b->d_tiles[st] = nullptr;
        b->ntiles[st] = (int)tiles[st].size();
        BCK(cudaMalloc(&b->d_tiles[st], sizeof(TileRef) * tiles[st].size()));
        BCK(cudaMemcpyAsync(b->d_tiles[st], tiles[st].data(), sizeof(TileRef) * tiles[st].size(),
                            cudaMemcpyHostToDevice, b->stream));
    }
    BCK(cudaStreamSynchronize(b->stream));
    b->dirty = false;
    return RMHD2D_OK;
}

void batch_enqueue_step(rmhd2d_batch *b, int parity)
{
    auto launch = batch_launcher(b->precision);
    const int n = (int)b->runs.size();
    const int ctas = b->nsm * b->ctas_per_sm;
    launch(1, b->shape, b->d_runs, b->d_maps, b->d_tiles[0], b->ntiles[0], ctas, parity, b->stream);
    launch_boundary_batch(b->d_runs, n, b->max_ghost, 0, 0, b->stream);
    launch(2, b->shape, b->d_runs, b->d_maps, b->d_tiles[1], b->ntiles[1], ctas, parity, b->stream);
    launch_boundary_batch(b->d_runs, n, b->max_ghost, 1, parity ^ 1, b->stream);
}

void batch_advance(rmhd2d_batch *b, int nsteps)
{
    b->steps += nsteps;
    if (nsteps & 1) b->parity ^= 1;
    for (auto *s : b->runs) {
        s->parity = b->parity;
        s->steps += nsteps;
    }
}

}  // namespace

extern "C" {

int rmhd2d_batch_create(const rmhd2d_config *cfgs, int nruns, rmhd2d_batch **out)
{
    rmhd2d_batch *b = nullptr;
    if (!cfgs || !out || nruns <= 0) return bfail(b, RMHD2D_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    for (int r = 1; r < nruns; ++r)
        if (cfgs[r].precision != cfgs[0].precision || cfgs[r].device != cfgs[0].device)
            return bfail(b, RMHD2D_ERR_INVALID, "all runs of a batch share precision and device");
    for (int r = 0; r < nruns; ++r)
        if (cfgs[r].ct_scheme != RMHD2D_CT_STAGE1)
            return bfail(b, RMHD2D_ERR_INVALID, "batched runs use the stage-1-EMF step (ct_scheme 0)");
    b = new rmhd2d_batch();
    b->device = cfgs[0].device;
    b->precision = cfgs[0].precision;
    auto bail = [&](int code, const std::string &msg) {
        {
            std::lock_guard<std::mutex> lk(g_err_mu);
            g_create_err = msg;
        }
        rmhd2d_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) return bail(RMHD2D_ERR_NO_DEVICE, "cudaSetDevice failed");
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, b->device) == cudaSuccess) b->nsm = prop.multiProcessorCount;
    if (cfgs[0].stream) {
        b->stream = (cudaStream_t)cfgs[0].stream;
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(RMHD2D_ERR_CUDA, "cudaStreamCreate failed");
        b->own_stream = true;
    }
    for (int r = 0; r < nruns; ++r) {
        rmhd2d_config c = cfgs[r];
        c.stream = b->stream;
        rmhd2d_solver *s = nullptr;
        const int rc = rmhd2d_create(&c, &s);
        if (rc) return bail(rc, std::string("run ") + std::to_string(r) + ": " + rmhd2d_last_error(nullptr));
        s->batch = b;
        b->runs.push_back(s);
    }
    *out = b;
    return RMHD2D_OK;
}

int rmhd2d_batch_destroy(rmhd2d_batch *b)
{
    if (!b) return RMHD2D_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    for (auto *s : b->runs) {
        s->batch = nullptr;
        destroy_solver(s);
    }
    cudaFree(b->d_runs);
    cudaFree(b->d_maps);
    cudaFree(b->d_tiles[0]);
    cudaFree(b->d_tiles[1]);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return RMHD2D_OK;
}

int rmhd2d_batch_size(const rmhd2d_batch *b, int *nruns)
{
    if (!b || !nruns) return RMHD2D_ERR_INVALID;
    *nruns = (int)b->runs.size();
    return RMHD2D_OK;
}

int rmhd2d_batch_member(rmhd2d_batch *b, int run, rmhd2d_solver **out)
{
    if (!b || !out) return bfail(b, RMHD2D_ERR_INVALID, "null argument");
    if (run < 0 || run >= (int)b->runs.size()) return bfail(b, RMHD2D_ERR_INVALID, "run index out of range");
    *out = b->runs[run];
    // state, eta tables or shape may change through the member: rebuild on the next step
    b->dirty = true;
    return RMHD2D_OK;
}

int rmhd2d_batch_set_launch(rmhd2d_batch *b, int shape, int ctas_per_sm)
{
    if (!b) return bfail(b, RMHD2D_ERR_INVALID, "null batch");
    if (shape < 0 || shape >= NSHAPE || ctas_per_sm < 1 || ctas_per_sm > shape_max_ctas(shape))
        return bfail(b, RMHD2D_ERR_INVALID, "tile shape must be 0..2 and CTAs per SM 1..2 (1 for shape 2)");
    b->shape = shape;
    b->ctas_per_sm = ctas_per_sm;
    b->dirty = true;
    return RMHD2D_OK;
}

int rmhd2d_batch_get_launch(const rmhd2d_batch *b, int *shape, int *ctas_per_sm)
{
    if (!b) return RMHD2D_ERR_INVALID;
    if (shape) *shape = b->shape;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    return RMHD2D_OK;
}

int rmhd2d_batch_run(rmhd2d_batch *b, int nsteps)
{
    if (!b) return bfail(b, RMHD2D_ERR_INVALID, "null batch");
    if (nsteps < 0) return bfail(b, RMHD2D_ERR_INVALID, "nsteps < 0");
    BCK(cudaSetDevice(b->device));
    int rc = batch_build(b);
    if (rc) return rc;
    // the two-step graphs of both step parities, captured together on first
    // use (as for a single solver, rmhd2d_run) and uploaded
    for (int p = 0; p < 2 && nsteps >= 2; ++p) {
        cudaGraphExec_t &ge = b->graph2[p];
        if (ge) continue;
        cudaGraph_t graph = nullptr;
        BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        batch_enqueue_step(b, p);
        batch_enqueue_step(b, p ^ 1);
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (e != cudaSuccess) return bfail(b, RMHD2D_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ge = nullptr;
            return bfail(b, RMHD2D_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        BCK(cudaGraphUpload(ge, b->stream));
    }
    while (nsteps >= 2) {
        BCK(cudaGraphLaunch(b->graph2[b->parity], b->stream));
        batch_advance(b, 2);
        nsteps -= 2;
    }
    if (nsteps == 1) {
        batch_enqueue_step(b, b->parity);
        BCK(cudaGetLastError());
        batch_advance(b, 1);
    }
    return RMHD2D_OK;
}

int rmhd2d_batch_run_timed(rmhd2d_batch *b, int nsteps, float *ms)
{
    if (!b || !ms) return bfail(b, RMHD2D_ERR_INVALID, "null argument");
    BCK(cudaSetDevice(b->device));
    int rc = batch_build(b);
    if (rc) return rc;
    ScopedEvent e0, e1;
    BCK(cudaEventCreate(&e0.e));
    BCK(cudaEventCreate(&e1.e));
    BCK(cudaEventRecord(e0.e, b->stream));
    rc = rmhd2d_batch_run(b, nsteps);
    if (rc) return rc;
    BCK(cudaEventRecord(e1.e, b->stream));
    BCK(cudaEventSynchronize(e1.e));
    BCK(cudaEventElapsedTime(ms, e0.e, e1.e));
    for (auto *s : b->runs) {
        const int r2 = sync_and_check(s);
        if (r2) return bfail(b, r2, rmhd2d_last_error(s));
    }
    return RMHD2D_OK;
}

int rmhd2d_batch_autotune(rmhd2d_batch *b, int trial_steps, int *best_shape, int *best_ctas_per_sm)
{
    if (!b) return bfail(b, RMHD2D_ERR_INVALID, "null batch");
    if (trial_steps < 2) trial_steps = 2;
    trial_steps += trial_steps & 1;   // even: the step parity comes back
    BCK(cudaSetDevice(b->device));
    std::vector<Snapshot> sn(b->runs.size());
    for (size_t r = 0; r < b->runs.size(); ++r) {
        const int rc = snapshot_take(b->runs[r], sn[r]);
        if (rc) return bfail(b, rc, rmhd2d_last_error(b->runs[r]));
    }
    const int par0 = b->parity;
    const long long steps0 = b->steps;
    float best = 1e30f;
    int bs = b->shape, bc = b->ctas_per_sm, rc = RMHD2D_OK;
    b->tune_shape.clear();
    b->tune_ctas.clear();
    b->tune_ms.clear();
    for (int sh = 0; sh < NSHAPE && !rc; ++sh)
        for (int c = 1; c <= shape_max_ctas(sh) && !rc; ++c) {
            rc = rmhd2d_batch_set_launch(b, sh, c);
            float warm = 0.f, ms = 0.f;
            if (!rc) rc = rmhd2d_batch_run_timed(b, 2, &warm);
            if (!rc) rc = rmhd2d_batch_run_timed(b, trial_steps, &ms);
            if (!rc) {
                b->tune_shape.push_back(sh);
                b->tune_ctas.push_back(c);
                b->tune_ms.push_back(ms / trial_steps);
            }
            if (!rc && ms < best) {
                best = ms;
                bs = sh;
                bc = c;
            }
        }
    int rc_restore = RMHD2D_OK;
    for (size_t r = 0; r < b->runs.size(); ++r) {
        const int r2 = snapshot_restore(b->runs[r], sn[r]);
        if (r2 && !rc_restore) rc_restore = bfail(b, r2, rmhd2d_last_error(b->runs[r]));
    }
    b->parity = par0;
    b->steps = steps0;
    if (rc) return rc;
    if (rc_restore) return rc_restore;
    rc = rmhd2d_batch_set_launch(b, bs, bc);
    if (best_shape) *best_shape = bs;
    if (best_ctas_per_sm) *best_ctas_per_sm = bc;
    return rc;
}

int rmhd2d_batch_get_tuning(const rmhd2d_batch *b, int max, int *n, int *shapes, int *ctas_per_sm, float *ms_per_step)
{
    if (!b || !n) return bfail(const_cast<rmhd2d_batch *>(b), RMHD2D_ERR_INVALID, "null argument");
    const int k = (int)b->tune_ms.size();
    *n = k;
    for (int q = 0; q < k && q < max; ++q) {
        if (shapes) shapes[q] = b->tune_shape[q];
        if (ctas_per_sm) ctas_per_sm[q] = b->tune_ctas[q];
        if (ms_per_step) ms_per_step[q] = b->tune_ms[q];
    }
    return RMHD2D_OK;
}

const char *rmhd2d_batch_last_error(const rmhd2d_batch *b)
{
    if (b) return b->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_create_err.c_str();
}

}  // extern "C"

namespace {

// Restores the calling thread's current device on scope exit.
struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

int rmhd2d_calculate_dt_noalloc(const rmhd2d_config *cfg, const double *device_state, double *dt)
{
    rmhd2d_solver *s = nullptr;
    if (!cfg || !device_state || !dt) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (cfg->nx < 12 || cfg->ny < 12) return fail(s, RMHD2D_ERR_INVALID, "nx and ny must be >= 12 (3 ghosts per side)");
    const long long ncell = (long long)cfg->nx * cfg->ny;
    if (ncell > RMHD2D_NOALLOC_MAX_CELLS)
        return fail(s, RMHD2D_ERR_INVALID,
                    "nx*ny = " + std::to_string(ncell) + " cells is above RMHD2D_NOALLOC_MAX_CELLS (" +
                        std::to_string((long long)RMHD2D_NOALLOC_MAX_CELLS) +
                        "), the size of the no-allocation scratch; use rmhd2d_calculate_dt on a solver");
    if (!(cfg->dx > 0) || !(cfg->dy > 0)) return fail(s, RMHD2D_ERR_INVALID, "dx and dy must be positive");
    if (!(cfg->gamma_mhd > 1.0)) return fail(s, RMHD2D_ERR_INVALID, "gamma_mhd must be > 1");
    if (!(cfg->eta >= 0.0)) return fail(s, RMHD2D_ERR_INVALID, "eta must be >= 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device || cfg->device < 0)
        return fail(s, RMHD2D_ERR_NO_DEVICE, "no CUDA device with that ordinal");
    DeviceRestore restore;
    CK(cudaGetDevice(&restore.prev));
    if (restore.prev == cfg->device) restore.prev = -1;
    else CK(cudaSetDevice(cfg->device));
    int major = 0, minor = 0;
    CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cfg->device));
    CK(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, cfg->device));
    if (major != 10 || minor != 0) return fail(s, RMHD2D_ERR_NO_DEVICE, "librmhd2d is built for sm_100a (B200) only");
    const cudaStream_t st = static_cast<cudaStream_t>(cfg->stream);
    // The call ends with a synchronisation of its stream, which a capture
    // would turn into an error that invalidates the caller's whole graph:
    // refuse before enqueuing anything.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(s, RMHD2D_ERR_STATE, "rmhd2d_calculate_dt_noalloc: cfg->stream is being captured; the call "
                                         "synchronises its stream and cannot be captured");
    unsigned long long *scratch = nullptr;
    CK(noalloc_scratch(&scratch));
    double out = 0.0;
    CK(enqueue_dt_noalloc(device_state, ncell, cfg->gamma_mhd, cfg->dx, cfg->dy, cfg->eps, cfg->eta, cfg->cfl,
                          scratch, &out, st));
    CK(cudaStreamSynchronize(st));
    *dt = out;
    return RMHD2D_OK;
}

// ---- slabs of a single domain decomposed along x -----------------------------
//
// One slab per rank (or per solver): its own interior columns plus 3 halo
// columns on each side that borders another slab.  The host exchanges halo
// columns between neighbours and combines the CFL / NaN reductions across
// slabs; the library fills the ghost cells of walls and runs the stages.

int rmhd2d_create_slab(const rmhd2d_config *cfg, int sides, rmhd2d_solver **out)
{
    rmhd2d_solver *s = nullptr;
    if (!cfg || !out) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (sides & ~(RMHD2D_SLAB_LO | RMHD2D_SLAB_HI | RMHD2D_SLAB_ORIGIN))
        return fail(s, RMHD2D_ERR_INVALID, "unknown slab flags");
    if (!(sides & RMHD2D_SLAB_LO) && !(sides & RMHD2D_SLAB_ORIGIN))
        return fail(s, RMHD2D_ERR_INVALID, "a slab whose low x side is a wall is the first slab: set RMHD2D_SLAB_ORIGIN");
    if (cfg->ct_scheme != RMHD2D_CT_STAGE1)
        return fail(s, RMHD2D_ERR_INVALID, "slabs run the stage-1-EMF CT only");
    const int rc = rmhd2d_create(cfg, out);
    if (rc) return rc;
    (*out)->g.x_halo = sides & (RMHD2D_SLAB_LO | RMHD2D_SLAB_HI);
    (*out)->slab = sides | SLAB_CREATED;
    return RMHD2D_OK;
}

int rmhd2d_slab_halo_doubles(const rmhd2d_solver *s, long long *n)
{
    if (!s || !n) return fail(const_cast<rmhd2d_solver *>(s), RMHD2D_ERR_INVALID, "null argument");
    *n = (long long)NFIELD * 3 * s->g.pitch;
    return RMHD2D_OK;
}

static int slab_state(rmhd2d_solver *s, int state, double **p)
{
    if (state != 0 && state != 1) return fail(s, RMHD2D_ERR_INVALID, "state must be 0 (current) or 1 (stage 1)");
    *p = state == 0 ? s->A : s->B;
    return RMHD2D_OK;
}

int rmhd2d_slab_pack(rmhd2d_solver *s, int state, int side, double *dev_buf)
{
    if (!s || !dev_buf) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    if (side != 0 && side != 1) return fail(s, RMHD2D_ERR_INVALID, "side must be 0 (low x) or 1 (high x)");
    double *st = nullptr;
    int rc = slab_state(s, state, &st);
    if (rc) return rc;
    CK(cudaSetDevice(s->device));
    launch_slab_halo(s->g, st, dev_buf, side == 0 ? HALO : s->g.nx - 2 * HALO, 1, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int rmhd2d_slab_unpack(rmhd2d_solver *s, int state, int side, const double *dev_buf)
{
    if (!s || !dev_buf) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    if (side != 0 && side != 1) return fail(s, RMHD2D_ERR_INVALID, "side must be 0 (low x) or 1 (high x)");
    if (!(s->g.x_halo & (1 << side))) return fail(s, RMHD2D_ERR_STATE, "that side is a wall, not a halo");
    double *st = nullptr;
    int rc = slab_state(s, state, &st);
    if (rc) return rc;
    CK(cudaSetDevice(s->device));
    launch_slab_halo(s->g, st, const_cast<double *>(dev_buf), side == 0 ? 0 : s->g.nx - HALO, 0, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int rmhd2d_slab_stage(rmhd2d_solver *s, int stage)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    if (stage != 1 && stage != 2) return fail(s, RMHD2D_ERR_INVALID, "stage must be 1 or 2");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    StageArgs a{};
    a.g = s->g;
    a.eta = s->eta;
    a.row2 = s->g.bc_x == BC_SYMMETRIC ? s->row2 : nullptr;
    a.ctl = s->ctl;
    a.parity = s->parity;
    auto launch = stage_launcher(s->cfg.precision);
    if (stage == 1) {
        a.src = s->A;
        a.un = s->A;
        a.dst = s->B;
        launch(1, s->shape, &s->mapA[s->shape], &s->mapE1[s->shape], a, s->stream);
    } else {
        a.src = s->B;
        a.un = s->A;
        a.dst = s->A;
        launch(2, s->shape2, &s->mapB[s->shape2], &s->mapE2[s->shape2], a, s->stream);
    }
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int rmhd2d_slab_fill(rmhd2d_solver *s, int which)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    if (which < 0 || which > 2) return fail(s, RMHD2D_ERR_INVALID, "which must be 0, 1 or 2");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    if (which == 0) {
        if (s->g.bc_x == BC_SYMMETRIC) launch_snapshot_row2(s->g, s->A, s->row2, s->stream);
        launch_boundary(s->g, s->A, s->row2, nullptr, 0, s->stream);
    } else if (which == 1) {
        launch_boundary(s->g, s->B, s->row2, nullptr, 0, s->stream);
    } else {
        launch_boundary(s->g, s->A, s->row2, s->ctl, s->parity ^ 1, s->stream);
        s->parity ^= 1;
        s->steps += 1;
    }
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int rmhd2d_slab_refresh_rate(rmhd2d_solver *s)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    CK(cudaSetDevice(s->device));
    return refresh_rate(s);
}

int rmhd2d_slab_get_words(rmhd2d_solver *s, long long *dev_words)
{
    if (!s || !dev_words) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    CK(cudaSetDevice(s->device));
    // the domain's ghost column 0 of a periodic-x decomposition sits in the
    // first slab's low halo, which its neighbour has just filled
    if ((s->slab & RMHD2D_SLAB_ORIGIN) && (s->g.x_halo & 1))
        launch_slab_origin_column(s->g, s->A, s->ctl, s->parity, s->stream);
    launch_slab_words(s->ctl, s->parity, dev_words, 1, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

int rmhd2d_slab_set_words(rmhd2d_solver *s, const long long *dev_words)
{
    if (!s || !dev_words) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!(s->slab & SLAB_CREATED)) return fail(s, RMHD2D_ERR_STATE, "not a slab (rmhd2d_create_slab)");
    CK(cudaSetDevice(s->device));
    launch_slab_words(s->ctl, s->parity, const_cast<long long *>(dev_words), 0, s->stream);
    CK(cudaGetLastError());
    return RMHD2D_OK;
}

// ---- discrete adjoint -------------------------------------------------------

extern "C" int rmhd2d_run_fixed_dt(rmhd2d_solver *s, int nsteps, const double *host_dts)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "run_fixed_dt");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: step the batch");
    if (nsteps < 0 || (nsteps > 0 && !host_dts)) return fail(s, RMHD2D_ERR_INVALID, "bad nsteps or dts");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    if (nsteps == 0) return RMHD2D_OK;
    CK(cudaSetDevice(s->device));
    DeviceBuffer d;
    CK(cudaMalloc(&d.p, (size_t)nsteps * sizeof(double)));
    CK(cudaMemcpyAsync(d.p, host_dts, (size_t)nsteps * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    int rc = set_fixed_dt_mode(s, 1);
    if (rc) return rc;
    FixedDtScope fixed{s, true};
    for (int n = 0; n < nsteps; ++n) {
        // the stage kernels read the step's dt from d.p + n; CT-Contact's
        // pipeline reads the control block's dt_fixed
        if (s->contact) {
            CK(cudaMemcpyAsync(&s->ctl->dt_fixed, d.p + n, sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
            enqueue_step(s, s->parity);
        } else {
            enqueue_step(s, s->parity, nullptr, d.p + n);
        }
        s->parity ^= 1;
        s->steps += 1;
    }
    fixed.armed = false;
    rc = set_fixed_dt_mode(s, 0);
    if (rc) return rc;
    CK(cudaGetLastError());
    return sync_and_check(s);
}

extern "C" int rmhd2d_adjoint_forward(rmhd2d_solver *s, int nsteps, int checkpoint_interval)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->g.x_halo) return refuse_halo_slab(s, "adjoint_forward");
    if (s->batch) return fail(s, RMHD2D_ERR_STATE, "member of a batch: step the batch");
    if (!s->has_state) return fail(s, RMHD2D_ERR_STATE, "no state set");
    if (nsteps < 1) return fail(s, RMHD2D_ERR_INVALID, "nsteps must be >= 1");
    if ((s->g.bc_x != BC_PERIODIC && s->g.bc_x != BC_SYMMETRIC) || (s->g.bc_y != BC_PERIODIC && s->g.bc_y != BC_SYMMETRIC))
        return fail(s, RMHD2D_ERR_INVALID, "the discrete adjoint is implemented for periodic and symmetric walls");
    if (s->contact) return fail(s, RMHD2D_ERR_INVALID, "the discrete adjoint differentiates the stage-1-EMF step");
    CK(cudaSetDevice(s->device));
    // checkpoint_interval < 0: one segment holding every step's U^n and U*,
    // written by the forward run itself, so backward recomputes nothing
    const bool tape = checkpoint_interval < 0;
    int interval = tape ? nsteps : checkpoint_interval;
    if (interval <= 0) interval = (int)std::ceil(std::sqrt((double)nsteps));
    if (interval > nsteps) interval = nsteps;
    const int nseg = (nsteps + interval - 1) / interval;
    const Grid &g = s->g;
    const size_t sd = (size_t)g.plane * NFIELD;
    // keep the workspace of an earlier run when it is large enough
    AdjointWork *w = s->adj;
    if (w && (w->cap_seg < nseg || w->cap_interval < interval || w->cap_steps < nsteps)) {
        CK(cudaStreamSynchronize(s->stream));
        free_adjoint(w);
        w = s->adj = nullptr;
    }
    if (!w) {
        w = new AdjointWork();
        w->state_doubles = sd;
        auto alloc = [&](double **p, size_t n, bool zero) -> cudaError_t {
            cudaError_t e = cudaMalloc(p, n * sizeof(double));
            if (e == cudaSuccess && zero) e = cudaMemsetAsync(*p, 0, n * sizeof(double), s->stream);
            return e;
        };
        cudaError_t e = cudaSuccess;
        const size_t P = (size_t)g.plane;
        // checkpoints and segment states are written before they are read;
        // the adjoint planes are cleared once so their unused padding is 0
        if (e == cudaSuccess) e = alloc(&w->ckpt, (size_t)nseg * sd, false);
        if (e == cudaSuccess) e = alloc(&w->seg0, (size_t)interval * sd, false);
        if (e == cudaSuccess) e = alloc(&w->seg1, (size_t)interval * sd, false);
        for (double *&u : w->ub)
            if (e == cudaSuccess) e = alloc(&u, sd, true);
        if (e == cudaSuccess) e = alloc(&w->Q, 18 * P, true);
        if (e == cudaSuccess) e = alloc(&w->IF, 32 * P, true);
        if (e == cudaSuccess) e = alloc(&w->RJ, 6 * P, true);
        if (e == cudaSuccess) e = alloc(&w->tmp, 2 * P, true);
        if (e == cudaSuccess) e = alloc(&w->etab, P, true);
        if (e == cudaSuccess) e = alloc(&w->dts, (size_t)nsteps, false);
        if (e == cudaSuccess) e = alloc(&w->final_state, sd, false);
        if (e == cudaSuccess) e = alloc(&w->aos, (size_t)g.nx * g.ny * NFIELD, false);
        if (e != cudaSuccess) {
            free_adjoint(w);
            return fail(s, RMHD2D_ERR_CUDA, std::string("adjoint workspace allocation: ") + cudaGetErrorString(e));
        }
        w->cap_seg = nseg;
        w->cap_interval = interval;
        w->cap_steps = nsteps;
        s->adj = w;
    }
    w->recorded = false;
    w->nsteps = nsteps;
    w->interval = interval;
    w->nseg = nseg;
    w->tape = tape;
    if (tape) {
        // every step reads U^n from and writes U* and U^{n+1} into the
        // segment slots, through each slot's own tensor maps
        w->map0.resize(nsteps);
        w->map1.resize(nsteps);
        for (int k = 0; k < nsteps; ++k)
            if (!encode_state_map(&w->map0[k], g, w->seg0 + (size_t)k * sd, stage_ui(1, s->shape), shape_uj(s->shape)) ||
                !encode_state_map(&w->map1[k], g, w->seg1 + (size_t)k * sd, stage_ui(2, s->shape2), shape_uj(s->shape2)))
                return fail(s, RMHD2D_ERR_CUDA, "cuTensorMapEncodeTiled failed for the adjoint's trajectory slots");
        CK(cudaMemcpyAsync(w->seg0, s->A, sd * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
        for (int n = 0; n < nsteps; ++n) {
            const size_t o = (size_t)n * sd;
            double *next = n + 1 < nsteps ? w->seg0 + o + sd : s->A;
            enqueue_step_between(s, s->parity, w->seg0 + o, &w->map0[n], w->seg1 + o, &w->map1[n], next, w->dts + n,
                                 nullptr);
            s->parity ^= 1;
            s->steps += 1;
        }
    } else {
        for (int n = 0; n < nsteps; ++n) {
            if (n % interval == 0)
                CK(cudaMemcpyAsync(w->ckpt + (size_t)(n / interval) * sd, s->A, sd * sizeof(double),
                                   cudaMemcpyDeviceToDevice, s->stream));
            enqueue_step(s, s->parity, w->dts + n);
            s->parity ^= 1;
            s->steps += 1;
        }
    }
    CK(cudaMemcpyAsync(w->final_state, s->A, sd * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaGetLastError());
    int rc = sync_and_check(s);
    if (rc) return rc;
    w->dts_host.resize(nsteps);
    CK(cudaMemcpy(w->dts_host.data(), w->dts, (size_t)nsteps * sizeof(double), cudaMemcpyDeviceToHost));
    w->ctl_final = *s->ctl_host;
    w->recorded = true;
    return RMHD2D_OK;
}

extern "C" int rmhd2d_adjoint_dts(rmhd2d_solver *s, double *host_dts)
{
    if (!s || !host_dts) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (!s->adj || !s->adj->recorded)
        return fail(s, RMHD2D_ERR_STATE, "no recorded forward run (rmhd2d_adjoint_forward)");
    std::memcpy(host_dts, s->adj->dts_host.data(), s->adj->dts_host.size() * sizeof(double));
    return RMHD2D_OK;
}

extern "C" int rmhd2d_adjoint_backward(rmhd2d_solver *s, const double *host_seed, double *host_grad_state,
                                       double *host_grad_eta)
{
    if (!s || !host_seed || !host_grad_state) return fail(s, RMHD2D_ERR_INVALID, "null argument");
    if (s->g.x_halo) return refuse_halo_slab(s, "adjoint_backward");
    if (!s->adj || !s->adj->recorded)
        return fail(s, RMHD2D_ERR_STATE, "no recorded forward run (rmhd2d_adjoint_forward)");
    CK(cudaSetDevice(s->device));
    AdjointWork *w = s->adj;
    const Grid &g = s->g;
    const size_t sd = w->state_doubles, naos = (size_t)g.nx * g.ny * NFIELD;
    cudaStream_t st = s->stream;
    CK(cudaMemcpyAsync(w->aos, host_seed, naos * sizeof(double), cudaMemcpyHostToDevice, st));
    launch_aos_to_planes(g, w->aos, w->ub[0], st);
    CK(cudaMemsetAsync(w->etab, 0, (size_t)g.plane * sizeof(double), st));
    // tensor maps of the segment slots for the solver's tile shape (a kept
    // trajectory is read as it is: nothing is recomputed)
    if (!w->tape) {
        w->map0.resize(w->interval);
        w->map1.resize(w->interval);
        for (int k = 0; k < w->interval; ++k)
            if (!encode_state_map(&w->map0[k], g, w->seg0 + (size_t)k * sd, stage_ui(1, s->shape), shape_uj(s->shape)) ||
                !encode_state_map(&w->map1[k], g, w->seg1 + (size_t)k * sd, stage_ui(2, s->shape2), shape_uj(s->shape2)))
                return fail(s, RMHD2D_ERR_CUDA, "cuTensorMapEncodeTiled failed for the adjoint's segment states");
    }
    int rc = set_fixed_dt_mode(s, 1);
    if (rc) return rc;
    FixedDtScope fixed{s, true};
    int cur = 0;
    for (int seg = w->nseg - 1; seg >= 0; --seg) {
        const int n0 = seg * w->interval;
        const int n1 = std::min(n0 + w->interval, w->nsteps);
        // recompute the segment from its checkpoint with the recorded dts,
        // each step reading U^n from and writing U* and U^{n+1} into the
        // segment's slots (the last U^{n+1} is not needed: A takes it)
        if (!w->tape) {
            CK(cudaMemcpyAsync(w->seg0, w->ckpt + (size_t)seg * sd, sd * sizeof(double), cudaMemcpyDeviceToDevice,
                               st));
            for (int n = n0; n < n1; ++n) {
                const int k = n - n0;
                const size_t o = (size_t)k * sd;
                double *next = n + 1 < n1 ? w->seg0 + o + sd : s->A;
                enqueue_step_between(s, 0, w->seg0 + o, &w->map0[k], w->seg1 + o, &w->map1[k], next, nullptr,
                                     w->dts + n);
            }
        }
        // reverse sweep over the segment
        for (int n = n1 - 1; n >= n0; --n) {
            const size_t o = (size_t)(n - n0) * sd;
            const int mid = (cur + 1) % 3, nxt = (cur + 2) % 3;
            AdjStageArgs a{};
            a.g = g;
            a.eta = s->eta;
            a.Q = w->Q;
            a.IF = w->IF;
            a.RJ = w->RJ;
            a.tmp = w->tmp;
            a.etab = w->etab;
            a.dt = w->dts_host[n];
            launch_boundary_transpose(g, w->ub[cur], st);
            a.W = w->seg1 + o;
            a.Ub = w->ub[cur];
            a.UbStep = w->ub[cur];
            a.Ustage = w->ub[mid];
            a.Uin = w->ub[nxt];
            a.s = 0.5;
            a.stage = 2;
            launch_adjoint_stage(a, st);
            launch_boundary_transpose(g, w->ub[mid], st);
            a.W = w->seg0 + o;
            a.Ub = w->ub[mid];
            a.UbStep = w->ub[cur];
            a.Ustage = nullptr;
            a.s = 1.0;
            a.stage = 1;
            launch_adjoint_stage(a, st);
            cur = nxt;
        }
        CK(cudaGetLastError());
    }
    // the boundary applied when the initial state was set
    launch_boundary_transpose(g, w->ub[cur], st);
    launch_planes_to_aos(g, w->ub[cur], w->aos, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host_grad_state, w->aos, naos * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (host_grad_eta) {
        launch_plane_to_table(g, w->etab, w->aos, st);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(host_grad_eta, w->aos, (size_t)g.nx * g.ny * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    // back to the end of the forward run (its control block has use_fixed_dt off)
    CK(cudaMemcpyAsync(s->A, w->final_state, sd * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->ctl, &w->ctl_final, sizeof(Control), cudaMemcpyHostToDevice, st));
    fixed.armed = false;
    return sync_and_check(s);
}

extern "C" int rmhd2d_adjoint_release(rmhd2d_solver *s)
{
    if (!s) return fail(s, RMHD2D_ERR_INVALID, "null solver");
    if (s->adj) {
        CK(cudaSetDevice(s->device));
        CK(cudaStreamSynchronize(s->stream));
        free_adjoint(s->adj);
        s->adj = nullptr;
    }
    return RMHD2D_OK;
}
