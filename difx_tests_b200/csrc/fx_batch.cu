// fx_batch.cu -- many independent correlation jobs in grouped launches,
// replayed as one CUDA graph, with an autotuner for the F-stage FFT
// block size and the plain X-stage tile variant (include/fxcorr.h, fxc_batch_*).
//
// Each job owns an ordinary context (device input, delay table, spectra chunk,
// accumulators).  Per round r (spectra chunk r of every job that has one):
//   one k_fstage_batch launch per F group  {FFT length, npol, spectra precision, FFTs per CTA}
//   one k_xplain_batch launch per X group  {8-signal blocks, tile variant} (plain form, <= 64 signals),
//   then one k_xplain_reduce per job of the group cut into time segments (as its single-job path cuts it)
//   one X launch per remaining job: the FP16 tensor-core X stage, or the plain X stage of
//   more than 64 signals
// A grouped launch works through a task table (F: persistent CTAs striding over it; plain X:
// one CTA per task), so small and large jobs share the
// machine inside one launch.  The delay tables and baseline counts run first.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/fxcorr.h"
#include "fx_ctx.h"
#include "fx_internal.h"
#include "fx_kernels.h"

using namespace fx;

namespace {

struct FGroup {
    int nchan, npol, mode, tb;   // mode: the jobs' spectra layout (fxc_ctx::spec_mode)
    std::vector<int> jobs;
};
struct XGroup {
    int nsig8, alt;   // signal blocks of 8 (jobs with the same count share tile plans)
    std::vector<int> jobs;
};
enum LaunchKind { kFGroup = 0, kXGroup = 1, kXJob = 2, kXReduce = 3 };
struct Launch {       // one launch of the recorded sequence
    int kind;         // LaunchKind
    int group;        // F / X group, or the job of a kXJob / kXReduce launch
    size_t task_off;  // into d_tasks (int4)
    int ntask;
    int round;        // kXJob / kXReduce: the round (spectra chunk) whose X arguments it takes
};

thread_local int g_batch_cuda = 0;

#define FB_CK(call)                                                                       \
    do {                                                                                  \
        const cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                          \
            g_batch_cuda = (int)e_;                                                       \
            return e_ == cudaErrorMemoryAllocation ? FXC_ERR_NOMEM : FXC_ERR_CUDA;        \
        }                                                                                 \
    } while (0)

// plan-cache keys as the single-job contexts write them ("F" FP32 spectra, "H" FP16)
std::string fkey(int nchan, int npol, int mode)
{
    return std::string(mode == kSpecF16 ? "H " : "F ") + std::to_string(2 * nchan) + " " + std::to_string(npol);
}
std::string xkey(int nsig8) { return "X " + std::to_string(nsig8); }

}  // namespace

struct fxc_batch {
    std::vector<fxc_ctx*> ctx;
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::vector<FGroup> fg;
    std::vector<XGroup> xg;
    std::vector<int> job_fg, job_xg;   // job_xg -1: the job's X stage is its own launch
    std::vector<XArgs> xa_host;        // [nrounds][J], for the launches of one job
    int nrounds = 0;
    // device tables: FArgs [nrounds][J], XArgs [nrounds][J], tasks (int4) for every recorded launch
    FArgs* d_fargs = nullptr;
    XArgs* d_xargs = nullptr;
    int4* d_tasks = nullptr;
    size_t task_cap = 0;
    std::vector<Launch> launches;
    bool tables_valid = false;
    // graph
    bool use_graph = true;
    bool warmed = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static void drop_graph(fxc_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

static int nchunks(const fxc_ctx* c) { return (c->cfg.numffts + c->T - 1) / c->T; }

// Slots chunk r of a job uses: its FFTs rounded up to the X stage's depth, as the single-job path
// rounds them (the F stage writes zeros after the last FFT, the X stage reads no further)
static int chunk_span(const fxc_ctx* c, int r)
{
    const int nfft = std::min(c->T, c->cfg.numffts - r * c->T);
    return std::min(c->T, (nfft + 63) / 64 * 64);
}

// Builds the F/X argument tables and the task list of every launch.
static int build_tables(fxc_batch* b)
{
    drop_graph(b);   // a recorded graph holds the old table pointers
    const int J = (int)b->ctx.size();
    b->nrounds = 0;
    for (auto* c : b->ctx) b->nrounds = std::max(b->nrounds, nchunks(c));
    std::vector<FArgs> fa((size_t)b->nrounds * J);
    std::vector<XArgs> xa((size_t)b->nrounds * J);
    for (int j = 0; j < J; j++) {
        fxc_ctx* c = b->ctx[j];
        for (int r = 0; r < nchunks(c); r++) {
            FArgs a = ctx_fargs(c, c->d_in, c->pitch, c->ld);
            a.t_base = r * c->T;
            a.nfft = std::min(c->T, c->cfg.numffts - r * c->T);
            a.tspan = chunk_span(c, r);
            a.tb = b->fg[b->job_fg[j]].tb;
            fa[(size_t)r * J + j] = a;
        }
        XArgs x{};
        x.spec = c->d_spec;
        x.acc = c->d_acc;
        x.nsig = c->nsig;
        x.T = c->T;
        x.nchan = c->cfg.nchan;
        x.nsb = c->cfg.nsubband;
        x.rows = c->rows;
        x.alt = b->job_xg[j] >= 0 ? b->xg[b->job_xg[j]].alt : c->plan_alt;
        if (c->cfg.xmode == FXC_X_PLAIN_FP32) ctx_xsegments(c, x);   // the single-job path's cut
        for (int r = 0; r < nchunks(c); r++) {
            xa[(size_t)r * J + j] = x;
            xa[(size_t)r * J + j].ntk = chunk_span(c, r);
        }
    }
    b->xa_host = xa;
    std::vector<int4> tasks;
    b->launches.clear();
    for (int r = 0; r < b->nrounds; r++) {
        for (int g = 0; g < (int)b->fg.size(); g++) {
            const size_t off = tasks.size();
            const int tb = b->fg[g].tb;
            for (int j : b->fg[g].jobs) {
                const fxc_ctx* c = b->ctx[j];
                if (r >= nchunks(c)) continue;
                for (int sb = 0; sb < c->cfg.nsubband; sb++)
                    for (int ant = 0; ant < c->cfg.nant; ant++)
                        for (int t0 = 0; t0 < chunk_span(c, r); t0 += tb)
                            tasks.push_back(make_int4(r * J + j, sb, ant, t0));
            }
            if (tasks.size() > off) b->launches.push_back({kFGroup, g, off, (int)(tasks.size() - off), r});
        }
        for (int g = 0; g < (int)b->xg.size(); g++) {
            const size_t off = tasks.size();
            const int cg = xplain_channel_group(b->xg[g].nsig8 * 8, b->xg[g].alt);
            std::vector<int> segd;   // jobs of the group cut into time segments: a reduce each after it
            for (int j : b->xg[g].jobs) {
                const fxc_ctx* c = b->ctx[j];
                if (r >= nchunks(c)) continue;
                const XArgs& xj = xa[(size_t)r * J + j];
                const int nseg = xplain_segments_used(xj);
                for (int sb = 0; sb < c->cfg.nsubband; sb++)
                    for (int c0 = 0; c0 < c->cfg.nchan; c0 += cg)
                        for (int s = 0; s < nseg; s++) tasks.push_back(make_int4(r * J + j, sb, c0, s));
                if (nseg > 1) segd.push_back(j);
            }
            if (tasks.size() > off) b->launches.push_back({kXGroup, g, off, (int)(tasks.size() - off), r});
            for (int j : segd) b->launches.push_back({kXReduce, j, 0, 0, r});
        }
        for (int j = 0; j < J; j++)
            if (b->job_xg[j] < 0 && r < nchunks(b->ctx[j])) b->launches.push_back({kXJob, j, 0, 0, r});
    }
    FB_CK(cudaSetDevice(b->device));
    cudaFree(b->d_fargs);
    cudaFree(b->d_xargs);
    b->d_fargs = nullptr;
    b->d_xargs = nullptr;
    if (tasks.size() > b->task_cap) {
        cudaFree(b->d_tasks);
        b->d_tasks = nullptr;
        FB_CK(cudaMalloc(&b->d_tasks, tasks.size() * sizeof(int4)));
        b->task_cap = tasks.size();
    }
    FB_CK(cudaMalloc(&b->d_fargs, std::max<size_t>(1, fa.size()) * sizeof(FArgs)));
    FB_CK(cudaMalloc(&b->d_xargs, std::max<size_t>(1, xa.size()) * sizeof(XArgs)));
    FB_CK(cudaMemcpy(b->d_fargs, fa.data(), fa.size() * sizeof(FArgs), cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(b->d_xargs, xa.data(), xa.size() * sizeof(XArgs), cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(b->d_tasks, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice));
    b->tables_valid = true;
    return FXC_OK;
}

static int enqueue_launch(fxc_batch* b, const Launch& l)
{
    if (l.kind == kFGroup) {
        const FGroup& g = b->fg[l.group];
        FB_CK(launch_fstage_batch(g.nchan, g.npol, g.mode, g.tb, b->d_fargs, b->d_tasks + l.task_off, l.ntask,
                                  b->stream));
    } else if (l.kind == kXGroup) {
        const XGroup& g = b->xg[l.group];
        FB_CK(launch_xplain_batch(g.nsig8 * 8, g.alt, b->d_xargs, b->d_tasks + l.task_off, l.ntask, b->stream));
    } else if (l.kind == kXReduce) {
        FB_CK(launch_xplain_reduce(b->xa_host[(size_t)l.round * b->ctx.size() + l.group], b->stream));
    } else {
        fxc_ctx* c = b->ctx[l.group];
        const XArgs& x = b->xa_host[(size_t)l.round * b->ctx.size() + l.group];
        FB_CK(c->cfg.xmode != FXC_X_TC_FP16 ? launch_xplain(x, b->stream)
              : c->xf32                     ? launch_xtc32(x, c->d_err, c->nsm, b->stream)
                                            : launch_xtc(x, c->d_err, c->nsm, b->stream));
    }
    return FXC_OK;
}

// FFTs per CTA candidates of an F group: the F16 staging of tb FFTs must fit one CTA's shared memory
static bool tb_fits(const fxc_batch* b, const FGroup& g, int tb)
{
    if (g.mode != kSpecF16) return true;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device) != cudaSuccess) return false;
    return fstage_smem_bytes(g.nchan, g.mode, g.npol, tb) <= (size_t)optin;
}

// The whole subintegration of every job: delay tables + counts, then the rounds.
static int enqueue_all(fxc_batch* b)
{
    for (fxc_ctx* c : b->ctx) {
        FB_CK(launch_delay_table(c->d_delays, c->d_offs, nullptr, 0, c->cfg.nant, c->cfg.numffts, c->ld, c->F,
                                 (c->cfg.numffts - 1) * c->F, 1.0 / (2.0 * c->cfg.bw), c->d_dtab, c->d_vbits,
                                 b->stream));
        FB_CK(launch_counts(c->d_vbits, c->cfg.nant, c->ld / 32, c->d_counts, b->stream));
    }
    for (const Launch& l : b->launches) {
        const int st = enqueue_launch(b, l);
        if (st != FXC_OK) return st;
    }
    return FXC_OK;
}

extern "C" {

int fxc_batch_create(const fxc_config* cfgs, int njobs, fxc_batch** out)
{
    if (!cfgs || njobs < 1 || !out) return FXC_ERR_INVALID;
    *out = nullptr;
    for (int j = 0; j < njobs; j++)
        if ((cfgs[j].xmode != FXC_X_PLAIN_FP32 && cfgs[j].xmode != FXC_X_TC_FP16) || cfgs[j].window_ffts != 0 ||
            cfgs[j].iscomplex || (cfgs[j].fstage != FXC_F_AUTO && cfgs[j].fstage != FXC_F_FFT32))
            return FXC_ERR_UNSUPPORTED;
    fxc_batch* b = new fxc_batch();
    int st = FXC_OK;
    for (int j = 0; j < njobs && st == FXC_OK; j++) {
        fxc_ctx* c = nullptr;
        st = ctx_create(&cfgs[j], &c, false);
        if (st == FXC_OK) b->ctx.push_back(c);
    }
    if (st == FXC_OK) {
        b->device = b->ctx[0]->device;
        if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) st = FXC_ERR_CUDA;
        b->stream = b->own;
    }
    if (st != FXC_OK) {
        fxc_batch_destroy(b);
        return st;
    }
    // groups (plans from the cache file when present)
    const auto plans = plan_cache_load();
    for (int j = 0; j < njobs; j++) {
        const fxc_ctx* c = b->ctx[j];
        const int mode = c->spec_mode;   // the layout the job's X stage reads
        int g = -1;
        for (int k = 0; k < (int)b->fg.size(); k++)
            if (b->fg[k].nchan == c->cfg.nchan && b->fg[k].npol == c->cfg.npol && b->fg[k].mode == mode) g = k;
        if (g < 0) {
            const auto it = plans.find(fkey(c->cfg.nchan, c->cfg.npol, mode));
            b->fg.push_back({c->cfg.nchan, c->cfg.npol, mode, it != plans.end() ? it->second : 16, {}});
            g = (int)b->fg.size() - 1;
            while (b->fg[g].tb > 4 && !tb_fits(b, b->fg[g], b->fg[g].tb)) b->fg[g].tb /= 2;
        }
        b->fg[g].jobs.push_back(j);
        b->job_fg.push_back(g);
        if (c->cfg.xmode != FXC_X_PLAIN_FP32 || c->nsig > 64) {
            b->job_xg.push_back(-1);   // its own X launch
            continue;
        }
        const int n8 = (c->nsig + 7) / 8;
        int h = -1;
        for (int k = 0; k < (int)b->xg.size(); k++)
            if (b->xg[k].nsig8 == n8) h = k;
        if (h < 0) {
            const auto it = plans.find(xkey(n8));
            b->xg.push_back({n8, it != plans.end() ? it->second : 0, {}});
            h = (int)b->xg.size() - 1;
        }
        b->xg[h].jobs.push_back(j);
        b->job_xg.push_back(h);
    }
    *out = b;
    return FXC_OK;
}

void fxc_batch_destroy(fxc_batch* b)
{
    if (!b) return;
    if (!b->ctx.empty()) cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    cudaFree(b->d_fargs);
    cudaFree(b->d_xargs);
    cudaFree(b->d_tasks);
    if (b->own) cudaStreamDestroy(b->own);
    for (auto* c : b->ctx) fxc_destroy(c);
    delete b;
}

int fxc_batch_upload(fxc_batch* b, int job, const uint8_t* const* data)
{
    if (!b || job < 0 || job >= (int)b->ctx.size()) return FXC_ERR_INVALID;
    fxc_ctx* c = b->ctx[job];
    FB_CK(cudaSetDevice(b->device));
    FB_CK(cudaStreamSynchronize(b->stream));   // a replay in flight may still read the old input
    const int st = fxc_upload_input(c, data);
    if (st != FXC_OK) return st;
    return fxc_synchronize(c);
}

int fxc_batch_set_model(fxc_batch* b, int job, const double* delays, const double* offs)
{
    if (!b || job < 0 || job >= (int)b->ctx.size() || !delays || !offs) return FXC_ERR_INVALID;
    fxc_ctx* c = b->ctx[job];
    const int A = c->cfg.nant;
    for (int i = 0; i < 3 * A; i++)
        if (!std::isfinite(delays[i])) return FXC_ERR_INVALID;
    for (int i = 0; i < A; i++)
        if (!std::isfinite(offs[i])) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    FB_CK(cudaStreamSynchronize(b->stream));   // a replay in flight may still read the old model
    FB_CK(cudaMemcpy(c->d_delays, delays, 3 * sizeof(double) * A, cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(c->d_offs, offs, sizeof(double) * A, cudaMemcpyHostToDevice));
    c->model_valid = false;   // the context's own upload cache no longer describes d_delays
    return FXC_OK;
}

int fxc_batch_process(fxc_batch* b)
{
    if (!b) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    if (!b->tables_valid) {
        const int st = build_tables(b);
        if (st != FXC_OK) return st;
    }
    if (!b->use_graph || !b->warmed) {
        b->warmed = true;   // the first run is eager: it also sets every kernel's shared-memory limit
        return enqueue_all(b);
    }
    if (!b->exec) {
        FB_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int st = enqueue_all(b);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (st != FXC_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        FB_CK(e);
        b->graph = g;
        FB_CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    FB_CK(cudaGraphLaunch(b->exec, b->stream));
    return FXC_OK;
}

int fxc_batch_reset(fxc_batch* b)
{
    if (!b) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    for (fxc_ctx* c : b->ctx) {
        FB_CK(cudaMemsetAsync(c->d_acc, 0, c->acc_bytes, b->stream));
        FB_CK(cudaMemsetAsync(c->d_counts, 0, sizeof(int) * c->npair_ant, b->stream));
    }
    return FXC_OK;
}

int fxc_batch_synchronize(fxc_batch* b)
{
    if (!b) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    FB_CK(cudaStreamSynchronize(b->stream));
    return FXC_OK;
}

int fxc_batch_get_visibilities(fxc_batch* b, int job, float* vis, int* counts, int normalize)
{
    if (!b || job < 0 || job >= (int)b->ctx.size()) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    FB_CK(cudaStreamSynchronize(b->stream));
    return fxc_get_visibilities(b->ctx[job], vis, counts, normalize);
}

int fxc_batch_set_stream(fxc_batch* b, void* s)
{
    if (!b) return FXC_ERR_INVALID;
    b->stream = s ? (cudaStream_t)s : b->own;
    return FXC_OK;
}

int fxc_batch_use_graph(fxc_batch* b, int enable)
{
    if (!b) return FXC_ERR_INVALID;
    b->use_graph = enable != 0;
    return FXC_OK;
}

int fxc_batch_launch_count(fxc_batch* b)
{
    if (!b) return FXC_ERR_INVALID;
    if (!b->tables_valid) {
        FB_CK(cudaSetDevice(b->device));
        const int st = build_tables(b);
        if (st != FXC_OK) return st;
    }
    return 2 * (int)b->ctx.size() + (int)b->launches.size();
}

int fxc_batch_get_plan(fxc_batch* b, int job, int* fft_block, int* x_variant)
{
    if (!b || job < 0 || job >= (int)b->ctx.size()) return FXC_ERR_INVALID;
    if (fft_block) *fft_block = b->fg[b->job_fg[job]].tb;
    if (x_variant) *x_variant = b->job_xg[job] >= 0 ? b->xg[b->job_xg[job]].alt : b->ctx[job]->plan_alt;
    return FXC_OK;
}

int fxc_batch_autotune(fxc_batch* b, int reps)
{
    if (!b || reps < 1) return FXC_ERR_INVALID;
    FB_CK(cudaSetDevice(b->device));
    cudaEvent_t e0, e1;
    FB_CK(cudaEventCreate(&e0));
    FB_CK(cudaEventCreate(&e1));
    int st = FXC_OK;
    // time the round-0 launch of one group under each candidate plan
    auto time_group = [&](int kind, int g, float* ms) -> int {
        if (!b->tables_valid && (st = build_tables(b)) != FXC_OK) return st;
        for (const Launch& l : b->launches) {
            if (l.kind != kind || l.group != g) continue;
            if ((st = enqueue_launch(b, l)) != FXC_OK) return st;   // warm / sets attributes
            FB_CK(cudaEventRecord(e0, b->stream));
            for (int i = 0; i < reps; i++)
                if ((st = enqueue_launch(b, l)) != FXC_OK) return st;
            FB_CK(cudaEventRecord(e1, b->stream));
            FB_CK(cudaEventSynchronize(e1));
            FB_CK(cudaEventElapsedTime(ms, e0, e1));
            return FXC_OK;
        }
        *ms = 0.f;
        return FXC_OK;
    };
    for (int g = 0; g < (int)b->fg.size() && st == FXC_OK; g++) {
        int best = b->fg[g].tb;
        float best_ms = 1e30f;
        for (int tb : {8, 16, 32}) {
            if (!tb_fits(b, b->fg[g], tb)) continue;
            b->fg[g].tb = tb;
            b->tables_valid = false;
            float ms = 0.f;
            if ((st = time_group(kFGroup, g, &ms)) != FXC_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = tb;
            }
        }
        b->fg[g].tb = best;
    }
    for (int g = 0; g < (int)b->xg.size() && st == FXC_OK; g++) {
        int best = b->xg[g].alt;
        float best_ms = 1e30f;
        for (int alt : {0, 1}) {
            b->xg[g].alt = alt;
            b->tables_valid = false;
            float ms = 0.f;
            if ((st = time_group(kXGroup, g, &ms)) != FXC_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = alt;
            }
        }
        b->xg[g].alt = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->tables_valid = false;
    drop_graph(b);
    b->warmed = false;
    if (st != FXC_OK) return st;
    {
        std::vector<std::string> lines;
        for (const auto& g : b->fg) lines.push_back(fkey(g.nchan, g.npol, g.mode) + " " + std::to_string(g.tb));
        for (const auto& g : b->xg) lines.push_back(xkey(g.nsig8) + " " + std::to_string(g.alt));
        plan_cache_append(lines);
    }
    return fxc_batch_reset(b);
}

}  // extern "C"
