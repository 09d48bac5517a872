// dg_ctx.cuh -- the context behind the C ABI's dg_ctx handle and the internal
// helpers shared by the single-case entry points (dg_capi.cu) and the batched
// ensembles (dg_batch.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>
#include <vector>

#include "../../include/dg_b200.h"
#include "../host/mesh.h"
#include "../host/numerics.h"
#include "dg_stage.cuh"

namespace dgi {
constexpr int kMaxVariants = 48;  // launch variants per order (checked in prepare_variant)

// NVTX range named after a C-ABI call, for timelines of Nsight tools (a no-op
// when no tool is attached)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
}

struct dg_ctx {
    int device = 0, p = 0, nb = 0, ne = 0, flux = 0, precision = 0;
    // partitioned contexts: ne owned elements (the first ninterior share no
    // face with a ghost), ne_alloc = ne + ghosts element slots in every state
    // buffer, and the halo plan on the device as (element, face) pairs
    int ne_alloc = 0, ninterior = 0, nslices = 0;
    int2* d_halo_send = nullptr;
    int2* d_halo_recv = nullptr;
    std::vector<int> peer_rank, peer_offset, peer_count;
    double gamma = 1.4, R = 287.05;
    cudaStream_t stream = nullptr;
    double *d_U0 = nullptr, *d_Ua = nullptr, *d_Ub = nullptr, *d_acc = nullptr, *d_out = nullptr;
    int2* d_conn = nullptr;
    dgk::FaceRec* d_frec = nullptr;    // [ne][6] face records of the owned elements
    int* d_geo_class = nullptr;
    dgk::GeoDev* d_geo = nullptr;
    uint8_t* d_cmap = nullptr;
    double* d_X0 = nullptr;
    // general (trilinear) geometry (pm.general): the stage kernel's per-point
    // tables (see dgk::StageArgs) and the element nodes [ne][8][3]
    double *d_gjd = nullptr, *d_gnrm = nullptr, *d_gimm = nullptr, *d_gnodes = nullptr;
    double* d_gfsd = nullptr;  // FP32 residual on general geometry: see dgk::StageArgs::gfsd
    // launch option FX (orders that compile FX variants): the faces, listed by
    // the side whose point order their flux is stored in -- first the nface_inner
    // faces that touch an interior element (computed with the interior
    // elements, before the halo exchange ends), then the others -- and the
    // face kernel's fluxes [nface][5][(p+2)^2]
    int nface = 0, nface_inner = 0;
    int2* d_faces = nullptr;
    double* d_fflux = nullptr;
    // contexts without ghosts list their faces by their lower element
    // (face_key[i] = min(elemL, elemR) of face i, ascending), so that element
    // chunks [e0, e1) first need the contiguous faces with key in [e0, e1):
    // the RK4 graph may then run each stage as `chunks` face launches on a
    // second stream, each followed on the main stream by the stage launch of
    // its element chunk (dg_set_stage_chunks)
    std::vector<int> face_key;
    int chunks = 1;
    cudaStream_t stream2 = nullptr;
    std::vector<cudaEvent_t> chunk_ev;  // 4 stages x (chunks + 1)
    // tensor-core variants (kTC): the basis operator in its shared-memory layout
    uint16_t* d_tcop = nullptr;
    int variant_face_grid[dgi::kMaxVariants] = {};  // face kernel grid per FX variant
    double* d_partials = nullptr;
    unsigned* d_status = nullptr;
    int red_grid = 0;
    int variant = 0;                                // index into dgk::stage_variants(p)
    int variant_grid[dgi::kMaxVariants] = {};       // persistent grid per variant, 0 = not prepared
    dgk::StageTables stage_tab{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    dgh::PreparedMesh pm;
    // per geometry class: time-step factor (a case's dt in a batch, else 1)
    // and the FP32 residual's energy reference (0 on the FP64 path)
    std::vector<double> class_dtf, class_eref;
    dgh::Tables1D tab;
    unsigned status_accum = 0;
    std::string err;
};

namespace dgi {

// records msg in the context (or, for c == nullptr, in the thread's creation
// error) and returns code
int fail(dg_ctx* c, int code, const std::string& msg);

#define DG_CUDA(c, call)                                                                         \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return ::dgi::fail((c), DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// dg_create with an optional per-element tag (elements with different tags
// never share a geometry class, so each class can carry one case's time step)
// and an optional partition (ghost elements after the owned ones)
int create_ctx(const dg_case_desc* cd, const dg_mesh_desc* md, const int* elem_tag, const dg_part_desc* part,
               dg_ctx** out);
void destroy_ctx(dg_ctx* c);

int prepare_variant(dg_ctx* c, int v);
bool variant_matches(const dg_ctx* c, int v);
// the stage kernels' arguments for elements [e_begin, e_end) with the context's variant
void stage_args(const dg_ctx* c, int mode, const double* Us, const double* U0, double* out, double dt, int e_begin,
                int e_end, dgk::StageArgs& a);
// stage launch over the owned elements [e_begin, e_end) (e_end < 0: all)
int launch_stage(dg_ctx* c, int mode, const double* Us, const double* U0, double* out, double dt, int e_begin = 0,
                 int e_end = -1);
int check_status(dg_ctx* c);

// state of elements [e0, e0 + ne) between the host layout [ne][nb][5] and the
// device layout [ne][5][nb] (staged through d_out / d_Ub); synchronous
int upload_range(dg_ctx* c, const double* Uc, double* dst, int e0, int ne);
int download_range(dg_ctx* c, const double* src, double* Uc, int e0, int ne);

// kind 0: sum over [e0, e0+ne) of the squared error against an exact solution
// per variable; kind 1: kinetic energy (out5[0]); deterministic order
int run_reduce(dg_ctx* c, int kind, int ic_type, const double* data, int ndata, double t, double* out5, int e0, int ne,
               double gamma, double R);

// L2 projection of an initial condition onto elements [e0, e0+ne) of d_U0, on
// the device (queued on the context's stream)
int project_ic_device(dg_ctx* c, int ic_type, const double* data, int ndata, double t, double gamma, double R, int e0,
                      int ne);

// uploads the geometry classes with class_dtf / class_eref
int upload_geometry(dg_ctx* c, cudaStream_t s);

// mean of rE over a host state [ne][nb][5] (the FP32 residual's energy
// reference), 0 for an FP64 context
double energy_reference(const dg_ctx* c, const double* Uc, int ne);

}  // namespace dgi
