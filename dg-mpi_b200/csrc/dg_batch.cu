// dg_batch.cu -- batched ensembles: the dg_batch_* entry points of
// include/dg_b200.h.
//
// Cases that share (order, flux, gamma, gas constant) form a group.  A group
// is one dg_ctx over the disjoint union of its cases' meshes: the face-gather
// table never crosses a case boundary because every neighbour index comes
// from the case's own interior_faces, and the geometry classes are split per
// case (create_ctx's element tags) so that each class carries its case's time
// step as the factor dtf of the stage update.  One RK4 step of the ensemble is
// a CUDA graph holding, for every group, its four stage launches (run with
// dt = 1, so each element advances by its class's dtf), the groups one after
// the other: each launch is a persistent grid sized for the whole GPU, and
// grids of different orders run side by side contend for the same SMs (the
// 256-case ensemble ran 12 % slower with the groups as concurrent branches).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../host/case.h"
#include "dg_ctx.cuh"
#include "dg_ensemble.cuh"

namespace {

thread_local std::string g_batch_create_error;

struct BatchGroup {
    int order = 0, flux = 0;
    double gamma = 1.4, R = 1.0;
    std::vector<int> cases;        // case ids, in element order
    std::vector<int> class_case;   // owning case of each geometry class
    dg_ctx* ctx = nullptr;
    int own_variant = 0;           // the group's launch variant in per-group mode
    int ens_variant = -1;          // the variant of the ensemble launch's configuration (-1: none)
};

struct BatchCase {
    int group = 0, e0 = 0, ne = 0, order = 0;
    double dt = 0.0, volume = 0.0, eref = 0.0;
};

}  // namespace

struct dg_batch {
    int device = 0, precision = 0;
    std::vector<BatchGroup> groups;
    std::vector<BatchCase> cases;
    cudaStream_t stream = nullptr;       // the stream the step graph is launched on
    std::vector<cudaEvent_t> events;     // fork / join events of the capture
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool geo_dirty = true;               // time steps changed since the last upload
    bool single = false;                 // one ensemble launch per RK stage (else one per group)
    int* d_work = nullptr;               // ensemble launches' batch counters [8 launches][8 groups]
    unsigned status_accum = 0;
    std::string err;
};

namespace {

int bfail(dg_batch* b, int code, const std::string& msg)
{
    if (b) b->err = msg;
    else g_batch_create_error = msg;
    return code;
}

// forwards a group context's error message
int gfail(dg_batch* b, int code, const BatchGroup& g)
{
    return bfail(b, code, "group of order " + std::to_string(g.order) + ": " + g.ctx->err);
}

void drop_graph(dg_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

void release_batch(dg_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    drop_graph(b);
    cudaFree(b->d_work);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (auto& g : b->groups) dgi::destroy_ctx(g.ctx);
}

bool case_ok(const dg_batch* b, int c) { return b && c >= 0 && c < static_cast<int>(b->cases.size()); }

// per-class time steps and energy references of every group to the device;
// the previous graph launches have finished (every stepping call synchronises)
int upload_time_steps(dg_batch* b)
{
    if (!b->geo_dirty) return DG_OK;
    for (auto& g : b->groups) {
        for (size_t k = 0; k < g.class_case.size(); ++k) {
            g.ctx->class_dtf[k] = b->cases[g.class_case[k]].dt;
            g.ctx->class_eref[k] = b->cases[g.class_case[k]].eref;
        }
        const int rc = dgi::upload_geometry(g.ctx, g.ctx->stream);
        if (rc) return gfail(b, rc, g);
    }
    b->geo_dirty = false;
    return DG_OK;
}

// relative cost per DOF and stage of the ensemble configuration of each order
// (inverse of the measured rates of those variants), weighting the groups'
// block ranges
double ensemble_cost(int p, bool fp32)
{
    static const double r32[dgk::kMaxP + 1] = {5.2, 16.6, 28.4, 37.4, 40.3, 40.8};
    static const double r64[dgk::kMaxP + 1] = {3.8, 11.3, 22.0, 29.7, 28.2, 31.2};
    return 1.0 / (fp32 ? r32[p] : r64[p]);
}

// splits `total` blocks over the groups in proportion to w (at least one per
// group with work, at most cap[g]) into boundaries blk[0..n]
void split_blocks(const std::vector<double>& w, const std::vector<int>& cap, int total, int* blk)
{
    double W = 0.0;
    for (double x : w) W += x;
    blk[0] = 0;
    for (size_t g = 0; g < w.size(); ++g) {
        int n = cap[g] > 0 ? static_cast<int>(std::lround(total * (W > 0 ? w[g] / W : 0.0))) : 0;
        n = std::min(std::max(n, cap[g] > 0 ? 1 : 0), cap[g]);
        blk[g + 1] = blk[g] + n;
    }
}

// the step graph with one face launch and one stage launch per RK stage for
// all groups (dg_ensemble.cuh)
int prepare_ensemble_graph(dg_batch* b)
{
    const bool fp32 = b->precision == DG_PREC_MIXED_FP32;
    const dgk::EnsembleKernels K = dgk::ensemble_kernels(fp32);
    const int ng = static_cast<int>(b->groups.size());
    unsigned mask = 0;
    for (auto& g : b->groups) mask |= 1u << g.order;
    const size_t smem = K.stage_smem(mask), fsmem = K.face_smem(mask);
    cudaError_t ce = cudaFuncSetAttribute(K.stage, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (ce == cudaSuccess) ce = cudaFuncSetAttribute(K.stage, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (ce == cudaSuccess) ce = cudaFuncSetAttribute(K.face, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsmem);
    int sms = 0, per_sm = 0, fper_sm = 0;
    if (ce == cudaSuccess) ce = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    if (ce == cudaSuccess) ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, K.stage, dgk::kEnsThreads, smem);
    if (ce == cudaSuccess) ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fper_sm, K.face, dgk::kFaceThreads, fsmem);
    if (ce != cudaSuccess) return bfail(b, DG_ERR_CUDA, std::string("ensemble launch set-up: ") + cudaGetErrorString(ce));
    if (per_sm < 1 || fper_sm < 1) return bfail(b, DG_ERR_UNSUPPORTED, "ensemble kernels do not fit on an SM");
    // block ranges: stage blocks by DOF x cost, face blocks by face points
    std::vector<double> ws(ng), wf(ng);
    std::vector<int> cs(ng), cf(ng);
    bool any_face = false;
    for (int g = 0; g < ng; ++g) {
        const BatchGroup& gr = b->groups[g];
        int E = 1, fl = 0;
        dgk::ensemble_config(gr.order, fp32, E, fl);
        const double nb = gr.ctx->nb, m = gr.order + 2;
        ws[g] = gr.ctx->ne * nb * ensemble_cost(gr.order, fp32);
        cs[g] = (gr.ctx->ne + E - 1) / E;
        const bool fx = (fl & dgk::kFX) != 0;
        const int fb = dgk::face_batch_of(gr.order, fp32 ? 4 : 8);
        wf[g] = fx ? gr.ctx->nface * m * m : 0.0;
        cf[g] = fx ? (gr.ctx->nface + fb - 1) / fb : 0;
        any_face = any_face || (fx && gr.ctx->nface > 0);
    }
    dgk::EnsembleArgs sa{}, fa{};
    sa.ngroup = fa.ngroup = ng;
    split_blocks(ws, cs, sms * per_sm, sa.blk);
    split_blocks(wf, cf, sms * fper_sm, fa.blk);
    for (int g = 0; g < ng; ++g) sa.order[g] = fa.order[g] = b->groups[g].order;
    constexpr int kCounters = 8 * dgk::kEnsMaxGroups;  // [stage 0..3][face, stage][group]
    if (!b->d_work && cudaMalloc((void**)&b->d_work, kCounters * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        b->d_work = nullptr;
        return bfail(b, DG_ERR_NOMEM, "ensemble work counters");
    }
    ce = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return bfail(b, DG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    ce = cudaMemsetAsync(b->d_work, 0, kCounters * sizeof(int), b->stream);  // every step starts at zero
    const int modes[4] = {dgk::kModeRK1, dgk::kModeRK2, dgk::kModeRK3, dgk::kModeRK4};
    for (int s = 0; s < 4 && ce == cudaSuccess; ++s) {
        for (int g = 0; g < ng; ++g) {
            dg_ctx* c = b->groups[g].ctx;
            const double* in[4] = {c->d_U0, c->d_Ua, c->d_Ub, c->d_Ua};
            double* out[4] = {c->d_Ua, c->d_Ub, c->d_Ua, c->d_U0};
            dgi::stage_args(c, modes[s], in[s], c->d_U0, out[s], 1.0, 0, c->ne, sa.g[g]);
            fa.g[g] = sa.g[g];
            if (cf[g] == 0) fa.g[g].nface = 0;  // no face kernel in this group's configuration
        }
        fa.work = b->d_work + (2 * s) * dgk::kEnsMaxGroups;
        sa.work = b->d_work + (2 * s + 1) * dgk::kEnsMaxGroups;
        if (any_face) ce = K.launch_face(fa, fa.blk[ng], fsmem, b->stream);
        if (ce == cudaSuccess) ce = K.launch_stage(sa, sa.blk[ng], smem, b->stream);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce_end = cudaStreamEndCapture(b->stream, &graph);
    if (ce != cudaSuccess || ce_end != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return bfail(b, DG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ce_end));
    }
    b->graph = graph;
    ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (ce != cudaSuccess) {
        drop_graph(b);
        return bfail(b, DG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    return DG_OK;
}

// the variant of group g's order with the ensemble launch's configuration, or -1
int ensemble_variant(const BatchGroup& g)
{
    const dg_ctx* c = g.ctx;
    if (c->p < 1 || c->pm.general) return -1;
    int E = 1, fl = 0;
    dgk::ensemble_config(c->p, c->precision == DG_PREC_MIXED_FP32, E, fl);
    const dgk::StageVariant* vs = nullptr;
    const int nv = dgk::stage_variants(c->p, &vs);
    for (int v = 0; v < nv; ++v)
        if (vs[v].E == E && vs[v].NT == dgk::kEnsThreads && vs[v].G == 1 && (vs[v].flags & 0xFF) == fl &&
            dgi::variant_matches(c, v))
            return v;
    return -1;
}

// one ensemble launch per RK stage (on = true), or one launch per group
int set_single_launch(dg_batch* b, bool on)
{
    if (on)
        for (auto& g : b->groups)
            if (g.ens_variant < 0)
                return bfail(b, DG_ERR_UNSUPPORTED, "group of order " + std::to_string(g.order) +
                                                        " has no launch variant for the ensemble launch (orders 1..5, affine meshes)");
    for (auto& g : b->groups) {
        const int v = on ? g.ens_variant : g.own_variant;
        const int rc = dg_set_stage_variant(g.ctx, v);
        if (rc) return gfail(b, rc, g);
    }
    if (on != b->single) drop_graph(b);
    b->single = on;
    return DG_OK;
}

int prepare_graph(dg_batch* b)
{
    if (b->exec) return DG_OK;
    if (b->single) return prepare_ensemble_graph(b);
    for (auto& g : b->groups) {
        const int rc = dgi::prepare_variant(g.ctx, g.ctx->variant);
        if (rc) return gfail(b, rc, g);
    }
    cudaError_t ce = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return bfail(b, DG_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    int rc = DG_OK;
    ce = cudaEventRecord(b->events[0], b->stream);
    for (size_t i = 0; i < b->groups.size() && ce == cudaSuccess && rc == DG_OK; ++i) {
        dg_ctx* c = b->groups[i].ctx;
        // a chain: group i starts when group i-1 has finished
        ce = cudaStreamWaitEvent(c->stream, b->events[i], 0);
        if (ce != cudaSuccess) break;
        rc = dgi::launch_stage(c, dgk::kModeRK1, c->d_U0, c->d_U0, c->d_Ua, 1.0);
        if (!rc) rc = dgi::launch_stage(c, dgk::kModeRK2, c->d_Ua, c->d_U0, c->d_Ub, 1.0);
        if (!rc) rc = dgi::launch_stage(c, dgk::kModeRK3, c->d_Ub, c->d_U0, c->d_Ua, 1.0);
        if (!rc) rc = dgi::launch_stage(c, dgk::kModeRK4, c->d_Ua, c->d_U0, c->d_U0, 1.0);
        if (rc) {
            rc = gfail(b, rc, b->groups[i]);
            break;
        }
        ce = cudaEventRecord(b->events[i + 1], c->stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->events[i + 1], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce_end = cudaStreamEndCapture(b->stream, &graph);
    if (rc != DG_OK || ce != cudaSuccess || ce_end != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        return bfail(b, DG_ERR_CUDA,
                     std::string("graph capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ce_end));
    }
    b->graph = graph;
    ce = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (ce != cudaSuccess) {
        drop_graph(b);
        return bfail(b, DG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    return DG_OK;
}

int check_groups(dg_batch* b)
{
    unsigned all = 0;
    for (auto& g : b->groups) {
        const int rc = dgi::check_status(g.ctx);
        if (rc == DG_ERR_NONPHYSICAL) {
            all |= g.ctx->status_accum;
            continue;
        }
        if (rc) return gfail(b, rc, g);
    }
    if (all) {
        b->status_accum |= all;
        char buf[160];
        snprintf(buf, sizeof(buf), "non-physical state detected on the device (status 0x%x)", all);
        return bfail(b, DG_ERR_NONPHYSICAL, buf);
    }
    return DG_OK;
}

// device time of `reps` RK4 steps of the batch in its current launch mode;
// every group's step-start state is saved before and restored after
int time_steps(dg_batch* b, int reps, float* ms)
{
    int rc = upload_time_steps(b);
    if (!rc) rc = prepare_graph(b);
    if (rc) return rc;
    cudaError_t ce = cudaSuccess;
    for (auto& g : b->groups) {
        const size_t bytes = static_cast<size_t>(g.ctx->ne_alloc) * g.ctx->nb * 5 * sizeof(double);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(g.ctx->d_out, g.ctx->d_U0, bytes, cudaMemcpyDeviceToDevice, b->stream);
    }
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (ce == cudaSuccess) ce = cudaEventCreate(&ev[0]);
    if (ce == cudaSuccess) ce = cudaEventCreate(&ev[1]);
    if (ce == cudaSuccess) ce = cudaGraphLaunch(b->exec, b->stream);  // warm-up step
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[0], b->stream);
    for (int r = 0; r < reps && ce == cudaSuccess; ++r) ce = cudaGraphLaunch(b->exec, b->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], b->stream);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(ms, ev[0], ev[1]);
    for (auto& g : b->groups) {
        const size_t bytes = static_cast<size_t>(g.ctx->ne_alloc) * g.ctx->nb * 5 * sizeof(double);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(g.ctx->d_U0, g.ctx->d_out, bytes, cudaMemcpyDeviceToDevice, b->stream);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->stream);
    if (ev[0]) cudaEventDestroy(ev[0]);
    if (ev[1]) cudaEventDestroy(ev[1]);
    if (ce != cudaSuccess) return bfail(b, DG_ERR_CUDA, std::string("dg_batch_tune timing: ") + cudaGetErrorString(ce));
    return check_groups(b);
}

}  // namespace

extern "C" {

int dg_batch_create(int ncases, const dg_case_desc* cases, const dg_mesh_desc* meshes, dg_batch** out)
{
    g_batch_create_error.clear();
    if (!out) return bfail(nullptr, DG_ERR_ARG, "dg_batch_create: null output");
    *out = nullptr;
    if (ncases < 1 || !cases || !meshes) return bfail(nullptr, DG_ERR_ARG, "dg_batch_create: no cases");
    for (int c = 0; c < ncases; ++c) {
        const dg_case_desc& cd = cases[c];
        const std::string tag = "case " + std::to_string(c) + ": ";
        if (cd.device != cases[0].device) return bfail(nullptr, DG_ERR_ARG, tag + "all cases must use one device");
        if (cd.precision != cases[0].precision) return bfail(nullptr, DG_ERR_ARG, tag + "all cases must use one precision");
        if (cd.order < 0 || cd.order > dgk::kMaxP) return bfail(nullptr, DG_ERR_UNSUPPORTED, tag + "order must be 0..5");
        if (cd.flux != DG_FLUX_LAX_FRIEDRICHS && cd.flux != DG_FLUX_HLLC) return bfail(nullptr, DG_ERR_ARG, tag + "unknown flux");
        if (!(cd.gamma > 1.0)) return bfail(nullptr, DG_ERR_ARG, tag + "gamma must exceed 1");
        const dg_mesh_desc& md = meshes[c];
        if (md.nelem <= 0 || md.nnode <= 0 || md.nface <= 0 || !md.node_coords || !md.elem_to_node_ids ||
            !md.interior_faces)
            return bfail(nullptr, DG_ERR_ARG, tag + "mesh arrays missing or empty");
        // each case's mesh on its own: the same checks and messages as dg_create
        dgh::MeshView mv;
        mv.nnode = md.nnode;
        mv.nelem = md.nelem;
        mv.nface = md.nface;
        mv.rank = md.rank;
        mv.coords = md.node_coords;
        mv.e2n = md.elem_to_node_ids;
        mv.faces = md.interior_faces;
        dgh::PreparedMesh pm;
        std::string perr;
        try {
            perr = dgh::prepare_mesh(mv, cd.order + 2, pm);
        } catch (const std::exception& ex) {
            perr = std::string("mesh preparation failed: ") + ex.what();
        }
        if (perr.empty() && pm.general)
            perr = "unsupported: non-affine elements (general geometry runs in single-case contexts)";
        if (!perr.empty())
            return bfail(nullptr, perr.rfind("unsupported:", 0) == 0 ? DG_ERR_UNSUPPORTED : DG_ERR_ARG, tag + perr);
    }

    dg_batch* b = new (std::nothrow) dg_batch();
    if (!b) return bfail(nullptr, DG_ERR_NOMEM, "host allocation failed");
    b->device = cases[0].device;
    b->precision = cases[0].precision;
    b->cases.resize(ncases);
    std::map<std::tuple<int, int, double, double>, int> group_of;
    for (int c = 0; c < ncases; ++c) {
        const auto key = std::make_tuple(cases[c].order, cases[c].flux, cases[c].gamma, cases[c].gas_constant);
        auto it = group_of.find(key);
        if (it == group_of.end()) {
            it = group_of.emplace(key, static_cast<int>(b->groups.size())).first;
            BatchGroup g;
            g.order = cases[c].order;
            g.flux = cases[c].flux;
            g.gamma = cases[c].gamma;
            g.R = cases[c].gas_constant;
            b->groups.push_back(g);
        }
        b->groups[it->second].cases.push_back(c);
        b->cases[c].group = it->second;
        b->cases[c].order = cases[c].order;
    }

    auto bail = [&](int code, const std::string& msg) {
        release_batch(b);
        delete b;
        return bfail(nullptr, code, msg);
    };
    // one context per group over the concatenated meshes
    for (auto& g : b->groups) {
        long long nnode = 0, nelem = 0, nface = 0;
        for (int c : g.cases) {
            nnode += meshes[c].nnode;
            nelem += meshes[c].nelem;
            nface += meshes[c].nface;
        }
        if (nelem > (1LL << 30) || nnode > (1LL << 31) - 1 || nface > (1LL << 31) - 1)
            return bail(DG_ERR_ARG, "group of order " + std::to_string(g.order) + " is too large");
        std::vector<double> coords(static_cast<size_t>(nnode) * 3);
        std::vector<unsigned> e2n(static_cast<size_t>(nelem) * 8), faces(static_cast<size_t>(nface) * 8);
        std::vector<int> tags(static_cast<size_t>(nelem));
        size_t no = 0, eo = 0, fo = 0;
        for (int c : g.cases) {
            const dg_mesh_desc& md = meshes[c];
            std::memcpy(&coords[no * 3], md.node_coords, static_cast<size_t>(md.nnode) * 3 * sizeof(double));
            for (size_t i = 0; i < static_cast<size_t>(md.nelem) * 8; ++i)
                e2n[eo * 8 + i] = md.elem_to_node_ids[i] + static_cast<unsigned>(no);
            for (size_t f = 0; f < static_cast<size_t>(md.nface); ++f) {
                const unsigned* r = md.interior_faces + f * 8;
                unsigned* w = &faces[(fo + f) * 8];
                // the ranks were checked per case; the group is one rank 0
                w[0] = 0; w[1] = r[1] + static_cast<unsigned>(eo); w[2] = r[2]; w[3] = r[3];
                w[4] = 0; w[5] = r[5] + static_cast<unsigned>(eo); w[6] = r[6]; w[7] = r[7];
            }
            for (int e = 0; e < md.nelem; ++e) tags[eo + e] = c;
            b->cases[c].e0 = static_cast<int>(eo);
            b->cases[c].ne = md.nelem;
            no += md.nnode;
            eo += md.nelem;
            fo += md.nface;
        }
        dg_mesh_desc gm{static_cast<int>(nnode), coords.data(), static_cast<int>(nelem), e2n.data(),
                        static_cast<int>(nface), faces.data(), 0};
        dg_case_desc gc = cases[g.cases[0]];
        const int rc = dgi::create_ctx(&gc, &gm, tags.data(), nullptr, &g.ctx);
        if (rc) return bail(rc, "group of order " + std::to_string(g.order) + ": " + dg_last_error(nullptr));
        const dgh::PreparedMesh& pm = g.ctx->pm;
        g.class_case.assign(pm.classes.size(), -1);
        for (size_t e = 0; e < tags.size(); ++e) g.class_case[pm.geo_class[e]] = tags[e];
        for (int c : g.cases) b->cases[c].volume = dgh::range_volume(pm, b->cases[c].e0, b->cases[c].e0 + b->cases[c].ne);
    }
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(DG_ERR_CUDA, "stream creation failed");
    b->events.assign(b->groups.size() + 1, nullptr);
    for (auto& e : b->events)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
            return bail(DG_ERR_CUDA, "event creation failed");
    int rc = upload_time_steps(b);
    if (rc) return bail(rc, b->err);
    // one ensemble launch per RK stage when every group has its configuration
    bool ens = true;
    for (auto& g : b->groups) {
        g.own_variant = g.ctx->variant;
        g.ens_variant = ensemble_variant(g);
        ens = ens && g.ens_variant >= 0;
    }
    // default: one launch per group (measured faster on the 256-case ensemble:
    // the single launch runs every order at the largest order's occupancy);
    // dg_batch_tune times both and keeps the faster
    (void)ens;
    *out = b;
    return DG_OK;
}

void dg_batch_destroy(dg_batch* b)
{
    if (!b) return;
    release_batch(b);
    delete b;
}

const char* dg_batch_last_error(const dg_batch* b) { return b ? b->err.c_str() : g_batch_create_error.c_str(); }

int dg_batch_num_groups(const dg_batch* b) { return b ? static_cast<int>(b->groups.size()) : 0; }

int dg_batch_group_info(const dg_batch* b, int g, int* order, int* ncases, int* nelem, int* variant)
{
    if (!b || g < 0 || g >= static_cast<int>(b->groups.size())) return DG_ERR_ARG;
    const BatchGroup& gr = b->groups[g];
    if (order) *order = gr.order;
    if (ncases) *ncases = static_cast<int>(gr.cases.size());
    if (nelem) *nelem = gr.ctx->ne;
    if (variant) *variant = gr.ctx->variant;
    return DG_OK;
}

int dg_batch_case_info(const dg_batch* b, int c, int* order, int* nelem, int* group, double* dt)
{
    if (!case_ok(b, c)) return DG_ERR_ARG;
    const BatchCase& k = b->cases[c];
    if (order) *order = k.order;
    if (nelem) *nelem = k.ne;
    if (group) *group = k.group;
    if (dt) *dt = k.dt;
    return DG_OK;
}

int dg_batch_set_state(dg_batch* b, int c, const double* Uc)
{
    if (!case_ok(b, c) || !Uc) return bfail(b, DG_ERR_ARG, "dg_batch_set_state: bad argument");
    BatchCase& k = b->cases[c];
    BatchGroup& g = b->groups[k.group];
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    const double e = dgi::energy_reference(g.ctx, Uc, k.ne);
    if (e != k.eref) {
        k.eref = e;
        b->geo_dirty = true;
    }
    const int rc = dgi::upload_range(g.ctx, Uc, g.ctx->d_U0, k.e0, k.ne);
    return rc ? gfail(b, rc, g) : DG_OK;
}

int dg_batch_get_state(dg_batch* b, int c, double* Uc)
{
    if (!case_ok(b, c) || !Uc) return bfail(b, DG_ERR_ARG, "dg_batch_get_state: bad argument");
    const BatchCase& k = b->cases[c];
    BatchGroup& g = b->groups[k.group];
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    const int rc = dgi::download_range(g.ctx, g.ctx->d_U0, Uc, k.e0, k.ne);
    return rc ? gfail(b, rc, g) : DG_OK;
}

int dg_batch_project_ic(dg_batch* b, int c, int ic_type, const double* data, int ndata, double t, double* Uc)
{
    dgi::NvtxRange nvtx_("dg_batch_project_ic");
    if (!case_ok(b, c)) return bfail(b, DG_ERR_ARG, "dg_batch_project_ic: case index out of range");
    if (ic_type < DG_IC_UNIFORM || ic_type > DG_IC_TAYLOR_GREEN) return bfail(b, DG_ERR_ARG, "unknown initial condition");
    const int need[] = {5, 0, 0, 9, 1};
    if (ndata < need[ic_type] || (ndata > 0 && !data)) return bfail(b, DG_ERR_ARG, "initial condition needs more data values");
    double d[16] = {0};
    for (int i = 0; i < ndata && i < 16; ++i) d[i] = data[i];
    BatchCase& k = b->cases[c];
    BatchGroup& g = b->groups[k.group];
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    int rc = dgi::project_ic_device(g.ctx, ic_type, d, 16, t, g.gamma, g.R, k.e0, k.ne);
    if (rc) return gfail(b, rc, g);
    const bool mixed = g.ctx->precision == DG_PREC_MIXED_FP32;
    if (!Uc && !mixed) {
        if (cudaStreamSynchronize(g.ctx->stream) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "projection failed");
        return DG_OK;
    }
    std::vector<double> tmp;
    double* host = Uc;
    if (!host) {
        tmp.resize(static_cast<size_t>(k.ne) * g.ctx->nb * 5);
        host = tmp.data();
    }
    rc = dgi::download_range(g.ctx, g.ctx->d_U0, host, k.e0, k.ne);
    if (rc) return gfail(b, rc, g);
    const double e = dgi::energy_reference(g.ctx, host, k.ne);
    if (e != k.eref) {
        k.eref = e;
        b->geo_dirty = true;
    }
    return DG_OK;
}

int dg_batch_cfl_time_step(dg_batch* b, int c, const double* Uc, double cfl, double* dt)
{
    if (!case_ok(b, c) || !Uc || !dt || !(cfl > 0.0)) return bfail(b, DG_ERR_ARG, "dg_batch_cfl_time_step: bad argument");
    const BatchCase& k = b->cases[c];
    const BatchGroup& g = b->groups[k.group];
    const double v = dgh::cfl_time_step(g.ctx->pm, g.order, g.gamma, Uc, cfl, k.e0, k.e0 + k.ne);
    if (!(v > 0.0)) return bfail(b, DG_ERR_NONPHYSICAL, "state has non-positive density or pressure");
    *dt = v;
    return DG_OK;
}

int dg_batch_set_time_step(dg_batch* b, int c, double dt)
{
    if (!case_ok(b, c) || !(dt >= 0.0) || !std::isfinite(dt)) return bfail(b, DG_ERR_ARG, "dg_batch_set_time_step: bad argument");
    if (b->cases[c].dt != dt) {
        b->cases[c].dt = dt;
        b->geo_dirty = true;
    }
    return DG_OK;
}

int dg_batch_rk4_steps_timed(dg_batch* b, int nsteps, double* device_ms)
{
    dgi::NvtxRange nvtx_("dg_batch_rk4_steps_timed");
    if (!b || nsteps < 0) return bfail(b, DG_ERR_ARG, "dg_batch_rk4_steps: bad argument");
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    int rc = upload_time_steps(b);
    if (!rc) rc = prepare_graph(b);
    if (rc) return rc;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t ce = cudaEventCreate(&ev[0]);
    if (ce == cudaSuccess) ce = cudaEventCreate(&ev[1]);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[0], b->stream);
    for (int s = 0; s < nsteps && ce == cudaSuccess; ++s) ce = cudaGraphLaunch(b->exec, b->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], b->stream);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    if (ev[0]) cudaEventDestroy(ev[0]);
    if (ev[1]) cudaEventDestroy(ev[1]);
    if (ce != cudaSuccess) return bfail(b, DG_ERR_CUDA, std::string("batched RK4: ") + cudaGetErrorString(ce));
    if (device_ms) *device_ms = ms;
    return check_groups(b);
}

int dg_batch_rk4_steps(dg_batch* b, int nsteps) { return dg_batch_rk4_steps_timed(b, nsteps, nullptr); }

int dg_batch_set_launch_mode(dg_batch* b, int single)
{
    if (!b) return DG_ERR_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    return set_single_launch(b, single != 0);
}

int dg_batch_get_launch_mode(const dg_batch* b) { return b ? (b->single ? 1 : 0) : -1; }

int dg_batch_tune(dg_batch* b, int reps)
{
    dgi::NvtxRange nvtx_("dg_batch_tune");
    if (!b || reps < 1) return bfail(b, DG_ERR_ARG, "dg_batch_tune: bad argument");
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    // each group's fastest variant, in per-group mode
    int rc = set_single_launch(b, false);
    if (rc) return rc;
    for (auto& g : b->groups) {
        const int keep = g.ctx->variant;
        int best = keep;
        rc = dg_tune_stage(g.ctx, reps, &best, nullptr);
        if (rc) return gfail(b, rc, g);
        g.own_variant = best;
        if (best != keep) drop_graph(b);
    }
    // then the launch mode: one launch per group against one launch per stage
    bool ens = true;
    for (auto& g : b->groups) ens = ens && g.ens_variant >= 0;
    if (!ens) return DG_OK;
    float ms_group = 0.f, ms_single = 0.f;
    if ((rc = time_steps(b, reps, &ms_group)) != DG_OK) return rc;
    if ((rc = set_single_launch(b, true)) != DG_OK) return rc;
    if ((rc = time_steps(b, reps, &ms_single)) != DG_OK) return rc;
    return ms_single < ms_group ? DG_OK : set_single_launch(b, false);
}

int dg_batch_l2_error(dg_batch* b, int c, int ic_type, const double* data, int ndata, double t, double* err)
{
    if (!case_ok(b, c) || !err) return bfail(b, DG_ERR_ARG, "dg_batch_l2_error: bad argument");
    if (ic_type < DG_IC_UNIFORM || ic_type > DG_IC_TAYLOR_GREEN) return bfail(b, DG_ERR_ARG, "unknown exact solution");
    const int need[] = {5, 0, 0, 9, 1};
    if (ndata < need[ic_type] || (ndata > 0 && !data)) return bfail(b, DG_ERR_ARG, "exact solution needs more data values");
    const BatchCase& k = b->cases[c];
    BatchGroup& g = b->groups[k.group];
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(b, DG_ERR_CUDA, "cudaSetDevice failed");
    double sums[5];
    const int rc = dgi::run_reduce(g.ctx, 0, ic_type, data, ndata, t, sums, k.e0, k.ne, g.gamma, g.R);
    if (rc) return gfail(b, rc, g);
    for (int v = 0; v < 5; ++v) err[v] = std::sqrt(sums[v] / k.volume);
    return DG_OK;
}

int dg_batch_status(dg_batch* b, unsigned* flags)
{
    if (!b || !flags) return bfail(b, DG_ERR_ARG, "dg_batch_status: null argument");
    unsigned all = b->status_accum;
    for (auto& g : b->groups) {
        unsigned f = 0;
        const int rc = dg_status(g.ctx, &f);
        if (rc) return gfail(b, rc, g);
        all |= f;
    }
    b->status_accum = 0;
    *flags = all;
    return DG_OK;
}

}  // extern "C"
