// edzt_host.cu — host runtime and C ABI of libedzt.
//
// The host side of the replaced Fortran entry points: per-context model and
// table caches, a device buffer pool, the batched-job runner that drives the
// persistent Lanczos kernel, the plain (one kernel per BLAS-1 step) engine
// used as the reference-structured GPU comparator, the drivers that restate
// ground_state / diag_lanczos / cluster_green_ftn / green_diag, and the
// extern "C" functions declared in include/edzt.h.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>
#include <atomic>
#include <algorithm>
#include <deque>
#include <thread>
#include <cuda_runtime.h>
#include "../../include/edzt.h"
#include "edzt_internal.h"
#include "tridiag.h"

namespace {


struct EdztError {
    int code;
    std::string msg;
};

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            throw EdztError{_e == cudaErrorMemoryAllocation ? EDZT_ERR_OOM : EDZT_ERR_CUDA,         \
                            std::string(#call) + ": " + cudaGetErrorString(_e)};                   \
    } while (0)

#define CKLAUNCH()                                                                                 \
    do {                                                                                           \
        cudaError_t _e = cudaGetLastError();                                                       \
        if (_e != cudaSuccess) throw EdztError{EDZT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(_e)}; \
    } while (0)

void arg_check(bool ok, const char* what)
{
    if (!ok) throw EdztError{EDZT_ERR_ARG, what};
}

// ---------------------------------------------------------------------------
// device memory pool (grow-only cache of cudaMalloc blocks, reused by size)
// ---------------------------------------------------------------------------
class Pool {
  public:
    ~Pool() { release_all(); }
    void* get(size_t bytes)
    {
        bytes = (bytes + 255) & ~(size_t)255;
        if (bytes == 0) bytes = 256;
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes) {
            void* p = it->second;
            used_[p] = it->first;
            free_.erase(it);
            return p;
        }
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            trim();
            e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw EdztError{EDZT_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed"};
            }
        }
        used_[p] = bytes;
        return p;
    }
    void put(void* p)
    {
        if (!p) return;
        auto it = used_.find(p);
        if (it == used_.end()) return;
        free_.emplace(it->second, p);
        used_.erase(it);
    }
    void trim()
    {
        for (auto& kv : free_) cudaFree(kv.second);
        free_.clear();
    }
    void release_all()
    {
        trim();
        for (auto& kv : used_) cudaFree(kv.first);
        used_.clear();
    }

  private:
    std::multimap<size_t, void*> free_;
    std::map<void*, size_t> used_;
};

// RAII lease of a pool block
template <class T>
struct Lease {
    Pool* pool = nullptr;
    T* p = nullptr;
    Lease() = default;
    Lease(Pool& pl, size_t n) : pool(&pl), p(static_cast<T*>(pl.get(n * sizeof(T)))) {}
    Lease(const Lease&) = delete;
    Lease& operator=(const Lease&) = delete;
    Lease(Lease&& o) noexcept : pool(o.pool), p(o.p) { o.p = nullptr; }
    Lease& operator=(Lease&& o) noexcept
    {
        if (this != &o) { reset(); pool = o.pool; p = o.p; o.p = nullptr; }
        return *this;
    }
    ~Lease() { reset(); }
    void reset()
    {
        if (p && pool) pool->put(p);
        p = nullptr;
    }
};

struct DevBuf {
    void* p = nullptr;
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { CK(cudaMalloc(&p, bytes > 0 ? bytes : 16)); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// True for memory the kernels of a context on `device` read directly: device
// memory of that GPU or managed memory.  Device memory of another GPU is an
// argument error (a kernel would fault on it without peer access); host
// memory, pinned or not, is staged through a copy.
bool is_device_ptr(const void* p, int device)
{
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeDevice && at.device != device)
        throw EdztError{EDZT_ERR_ARG, "vector argument is device memory of GPU " + std::to_string(at.device) +
                                          ", not of the context's GPU " + std::to_string(device)};
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------
struct StrTable {
    int n = 0, count = 0;
    std::unique_ptr<DevBuf> str, rank;
};

struct OpsTable {
    int hw = 0, namp = 0;
    std::unique_ptr<DevBuf> e1, hcnt, hpk, amp, imp, sub;
};

// The model-dependent tables of one impurity model: per-spin operator tables
// by (electron count, spin) and the interaction tables.  The single-model
// entry points use the context's own; a batch holds one per instance.
struct ModelTables {
    bool valid = false;
    DevModel model{};
    int P = 1;
    bool has_j = false;
    std::map<std::pair<int, int>, std::unique_ptr<OpsTable>> ops;
    std::unique_ptr<DevBuf> wint, jcnt, jt;
};

}  // namespace

struct edzt_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int engine = EDZT_ENGINE_FUSED;
    int diag_solver = EDZT_DIAG_LANCZOS;    // ground_state's diag_solver (ground_state.f90:53-60)
    int keep_vectors = 1;                   // ground_state: keep the scan's Lanczos vectors when they fit
    size_t free_at_create = 0;              // free device memory when the context was created
    ModelTables mt;                         // the model of the single-model entry points
    // bit strings and rank tables by (nsite, electron count): model-independent, shared
    std::map<std::pair<int, int>, std::unique_ptr<StrTable>> str_tables;
    Pool pool;
    // resident ground state
    bool has_gs = false;
    int gs_up = 0, gs_dn = 0, gs_isector = -1;
    double gs_e0 = 0.0, gs_residual = 0.0;
    Lease<double> gs_vec;
    // persistent-kernel scratch
    std::unique_ptr<DevBuf> sync_words, status;
    // persistent-kernel statistics
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    long long st_launches = 0;
    double st_ms = 0.0, st_bytes = 0.0;
    // small host-visible scratch for the plain engine
    double* pinned = nullptr;
    std::unique_ptr<DevBuf> scal;          // device scalars
    std::unique_ptr<DevBuf> dot_part;      // dot partials
    std::atomic<long long> launches{0};    // kernel launches issued by this context
    // fault-test settings (edzt_set_fault_test): pass cap, barrier wait limit, stalled CTA
    int dbg_pass_cap = 0;
    unsigned long long dbg_wait_ns = 0;
    int dbg_stall_cta = -1;
    // tile shapes chosen by edzt_tune_sector, by (up strings, down strings)
    struct Tuned { int wc, r, block; double ms_per_step; };
    std::map<std::pair<int, int>, Tuned> tuned;
    // per launch since the last statistics reset: device ms, algorithmic
    // bytes, states in the launch (the last kLaunchLog)
    std::vector<double> log_ms, log_bytes, log_states;
};

namespace {

int nsite_of(const edzt_ctx* c) { return c->mt.model.nsite; }

StrTable& str_table_ns(edzt_ctx* c, int ns, int n)
{
    const auto key = std::make_pair(ns, n);
    auto it = c->str_tables.find(key);
    if (it != c->str_tables.end()) return *it->second;
    auto t = std::make_unique<StrTable>();
    t->n = n;
    t->count = (int)edzt_binom(ns, n);
    t->str = std::make_unique<DevBuf>(sizeof(uint32_t) * (size_t)std::max(t->count, 1));
    t->rank = std::make_unique<DevBuf>(sizeof(int32_t) * ((size_t)1 << ns));
    launch_build_strings(ns, n, t->str->as<uint32_t>(), t->rank->as<int32_t>(), c->stream);
    c->launches += 2;
    CKLAUNCH();
    StrTable& ref = *t;
    c->str_tables.emplace(key, std::move(t));
    return ref;
}

StrTable& str_table(edzt_ctx* c, int n) { return str_table_ns(c, nsite_of(c), n); }

OpsTable& ops_table_mt(edzt_ctx* c, ModelTables& mt, int n, int sigma)
{
    auto key = std::make_pair(n, sigma);
    auto it = mt.ops.find(key);
    if (it != mt.ops.end()) return *it->second;
    StrTable& st = str_table_ns(c, mt.model.nsite, n);
    auto t = std::make_unique<OpsTable>();
    const int norb = mt.model.norb, nbath = mt.model.nbath;
    // hop slots per string: the largest hop count of any string, rounded up to whole uint4s
    const int maxh = edzt_max_hops(mt.model, sigma, n);
    t->hw = std::max(4, (maxh + 3) / 4 * 4);
    t->namp = std::max(2, 2 * norb * nbath);
    const size_t cnt = (size_t)std::max(st.count, 1);
    t->e1 = std::make_unique<DevBuf>(sizeof(double) * cnt);
    t->hcnt = std::make_unique<DevBuf>(cnt);
    t->hpk = std::make_unique<DevBuf>(sizeof(uint32_t) * cnt * t->hw);
    t->amp = std::make_unique<DevBuf>(sizeof(double) * t->namp);
    t->imp = std::make_unique<DevBuf>(cnt);
    if (mt.has_j) t->sub = std::make_unique<DevBuf>(sizeof(int32_t) * cnt * mt.P);
    launch_build_spin_ops(mt.model, sigma, st.count, st.str->as<uint32_t>(), st.rank->as<int32_t>(), t->hw,
                          t->e1->as<double>(), t->hcnt->as<uint8_t>(), t->hpk->as<uint32_t>(),
                          t->amp->as<double>(), t->imp->as<uint8_t>(), t->sub ? t->sub->as<int32_t>() : nullptr,
                          c->stream);
    c->launches += 1;
    CKLAUNCH();
    OpsTable& ref = *t;
    mt.ops.emplace(key, std::move(t));
    return ref;
}

bool sector_valid_ns(int ns, int nu, int nd) { return nu >= 0 && nd >= 0 && nu <= ns && nd <= ns; }

long long sector_dim_ns(int ns, int nu, int nd)
{
    if (!sector_valid_ns(ns, nu, nd)) return 0;
    return (long long)edzt_binom(ns, nu) * (long long)edzt_binom(ns, nd);
}

bool sector_valid(const edzt_ctx* c, int nu, int nd) { return sector_valid_ns(nsite_of(c), nu, nd); }

long long sector_dim(const edzt_ctx* c, int nu, int nd) { return sector_dim_ns(nsite_of(c), nu, nd); }

DevSector make_sector_mt(edzt_ctx* c, ModelTables& mt, int nu, int nd)
{
    DevSector S{};
    const int ns = mt.model.nsite;
    StrTable& su = str_table_ns(c, ns, nu);
    StrTable& sd = str_table_ns(c, ns, nd);
    OpsTable& ou = ops_table_mt(c, mt, nu, 0);
    OpsTable& od = ops_table_mt(c, mt, nd, 1);
    auto fill = [&](DevSpin& sp, StrTable& st, OpsTable& o) {
        sp.count = st.count;
        sp.hw = o.hw;
        sp.namp = o.namp;
        sp.str = st.str->as<uint32_t>();
        sp.rank = st.rank->as<int32_t>();
        sp.e1 = o.e1->as<double>();
        sp.hcnt = o.hcnt->as<uint8_t>();
        sp.hpk = o.hpk->as<uint4>();
        sp.amp = o.amp->as<double>();
        sp.imp = o.imp->as<uint8_t>();
        sp.sub = o.sub ? o.sub->as<int32_t>() : nullptr;
    };
    fill(S.up, su, ou);
    fill(S.dn, sd, od);
    S.dim = (long long)su.count * sd.count;
    arg_check(S.dim < (1LL << 32), "sector dimension must stay below 2^32 states");
    arg_check(hx_fits(su.count, sd.count),
              "sector too large for the shared-memory staging of H.v (more than 13,000 strings of a spin: "
              "beyond nsite 16 at half filling)");
    S.P = mt.P;
    S.has_j = mt.has_j ? 1 : 0;
    S.wint = mt.wint->as<double>();
    S.jcnt = mt.jcnt->as<int>();
    S.jt = mt.jt->as<JTrans>();
    return S;
}

DevSector make_sector(edzt_ctx* c, int nu, int nd) { return make_sector_mt(c, c->mt, nu, nd); }

// Interaction tables over impurity occupation patterns (pu, pd).
// wint: impurity_hamiltonian.f90:119-141 without the em-mu terms (those are
// one-body and live in e1).  Exchange transitions: :179-226.
void build_model_tables(ModelTables& mt, cudaStream_t stream)
{
    const DevModel& m = mt.model;
    const int norb = m.norb, P = 1 << norb;
    mt.P = P;
    std::vector<double> w(P * P, 0.0);
    std::vector<int> jc(P * P, 0);
    std::vector<JTrans> jt((size_t)P * P * EDZT_MAX_JT);
    bool any_j = false;
    for (int pu = 0; pu < P; pu++)
        for (int pd = 0; pd < P; pd++) {
            double e = 0.0;
            for (int a = 0; a < norb; a++) {
                const int n1 = (pu >> a) & 1, n2 = (pd >> a) & 1;
                e += m.U * n1 * n2;
                for (int b = a + 1; b < norb; b++) {
                    const int m1 = (pu >> b) & 1, m2 = (pd >> b) & 1;
                    e += (m.Up - m.Jex) * (n1 * m1 + n2 * m2) + m.Up * (n1 * m2 + n2 * m1);
                }
            }
            w[pu * P + pd] = e;
            int cnt = 0;
            if (m.Jp != 0.0) {
                for (int i = 1; i <= norb; i++)
                    for (int j = 1; j <= norb; j++) {
                        if (i == j) continue;
                        const int ni1 = (pu >> (i - 1)) & 1, ni2 = (pd >> (i - 1)) & 1;
                        const int nj1 = (pu >> (j - 1)) & 1, nj2 = (pd >> (j - 1)) & 1;
                        const int lo = std::min(i, j), hi = std::max(i, j);
                        int par = 0;
                        for (int k = lo; k <= hi - 1; k++) par += ((pu >> (k - 1)) & 1) + ((pd >> (k - 1)) & 1);
                        const double s2 = (par & 1) ? -1.0 : 1.0;
                        if (ni1 == 0 && nj1 != 0 && nj2 == 0 && ni2 != 0) {   // spin-flip :201-211
                            JTrans t;
                            t.pu2 = (pu & ~(1 << (j - 1))) | (1 << (i - 1));
                            t.pd2 = (pd & ~(1 << (i - 1))) | (1 << (j - 1));
                            t.c = -(s2 * m.Jp);
                            jt[((size_t)pu * P + pd) * EDZT_MAX_JT + cnt++] = t;
                        }
                        if (ni1 == 0 && ni2 == 0 && nj1 != 0 && nj2 != 0) {   // pair-hop :215-225
                            JTrans t;
                            t.pu2 = (pu & ~(1 << (j - 1))) | (1 << (i - 1));
                            t.pd2 = (pd & ~(1 << (j - 1))) | (1 << (i - 1));
                            t.c = s2 * m.Jp;
                            jt[((size_t)pu * P + pd) * EDZT_MAX_JT + cnt++] = t;
                        }
                    }
            }
            jc[pu * P + pd] = cnt;
            any_j = any_j || cnt > 0;
        }
    mt.has_j = any_j;
    mt.wint = std::make_unique<DevBuf>(sizeof(double) * P * P);
    mt.jcnt = std::make_unique<DevBuf>(sizeof(int) * P * P);
    mt.jt = std::make_unique<DevBuf>(sizeof(JTrans) * jt.size());
    CK(cudaMemcpyAsync(mt.wint->p, w.data(), sizeof(double) * P * P, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(mt.jcnt->p, jc.data(), sizeof(int) * P * P, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(mt.jt->p, jt.data(), sizeof(JTrans) * jt.size(), cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));      // the host vectors go out of scope
}

// The reference's em(norb,2), ek(nbath,2), vmk(norb,nbath,2) (column-major) as a DevModel.
DevModel model_from(int norb, int nbath, const double* em, const double* ek, const double* vmk, double U,
                    double Up, double Jex, double Jp, double mu)
{
    arg_check(norb >= 1 && norb <= EDZT_MAX_NORB, "norb must be in [1, 4]");
    arg_check(nbath >= 0 && norb + nbath <= EDZT_MAX_NSITE, "norb + nbath must be <= 20");
    arg_check(em != nullptr && (nbath == 0 || (ek != nullptr && vmk != nullptr)), "em/ek/vmk required");
    DevModel m{};
    m.norb = norb; m.nbath = nbath; m.nsite = norb + nbath;
    for (int s = 0; s < 2; s++) {
        for (int a = 0; a < norb; a++) m.em[a][s] = em[a + norb * s];
        for (int l = 0; l < nbath; l++) m.ek[l][s] = ek[l + nbath * s];
        for (int a = 0; a < norb; a++)
            for (int l = 0; l < nbath; l++) m.vmk[a][l][s] = vmk[a + norb * (l + nbath * s)];
    }
    m.U = U; m.Up = Up; m.Jex = Jex; m.Jp = Jp; m.mu = mu;
    bool finite = std::isfinite(U) && std::isfinite(Up) && std::isfinite(Jex) && std::isfinite(Jp) && std::isfinite(mu);
    for (int s = 0; s < 2; s++) {
        for (int a = 0; a < norb; a++) finite = finite && std::isfinite(m.em[a][s]);
        for (int l = 0; l < nbath; l++) finite = finite && std::isfinite(m.ek[l][s]);
        for (int a = 0; a < norb; a++)
            for (int l = 0; l < nbath; l++) finite = finite && std::isfinite(m.vmk[a][l][s]);
    }
    arg_check(finite, "model parameters must be finite");
    return m;
}

void set_tables_model(ModelTables& mt, const DevModel& m, cudaStream_t stream)
{
    mt.ops.clear();
    mt.model = m;
    build_model_tables(mt, stream);
    mt.valid = true;
}

// ---------------------------------------------------------------------------
// host <-> device argument staging
// ---------------------------------------------------------------------------
struct InVec {
    const double* d = nullptr;
    Lease<double> tmp;
    InVec(edzt_ctx* c, const double* p, long long n)
    {
        if (is_device_ptr(p, c->device)) { d = p; return; }
        tmp = Lease<double>(c->pool, (size_t)std::max(n, 1LL));
        if (n > 0) CK(cudaMemcpyAsync(tmp.p, p, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        d = tmp.p;
    }
};

struct OutVec {
    double* d = nullptr;
    double* host = nullptr;
    long long n = 0;
    Lease<double> tmp;
    edzt_ctx* c;
    OutVec(edzt_ctx* cc, double* p, long long nn) : n(nn), c(cc)
    {
        if (is_device_ptr(p, c->device)) { d = p; return; }
        host = p;
        tmp = Lease<double>(c->pool, (size_t)std::max(n, 1LL));
        d = tmp.p;
    }
    void preload()
    {   // accumulate semantics need the caller's values on the device
        if (host && n > 0) CK(cudaMemcpyAsync(d, host, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    }
    void finish()
    {
        if (host && n > 0) {
            CK(cudaMemcpyAsync(host, d, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
        }
    }
};

void copy_out(edzt_ctx* c, void* dst, const void* src, size_t bytes)
{
    if (!dst || bytes == 0) return;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
}

// ---------------------------------------------------------------------------
// batched persistent Lanczos
// ---------------------------------------------------------------------------
struct JobSpec {
    ModelTables* mt = nullptr;       // model of the run (nullptr: the context's)
    int nu = 0, nd = 0;
    int mode = LZ_COEFF;
    int init = LZ_INIT_HASH;
    uint64_t key = 0;
    ApplyCArgs ac{};
    const double* ac_src = nullptr;
    int maxnstep = 0;
    const double* coeff = nullptr;   // device, EIGVEC
    double* eig = nullptr;           // device, EIGVEC
    double* a = nullptr;             // device [maxnstep]
    double* b = nullptr;             // device [maxnstep]
    double2* keep = nullptr;         // device [maxnstep + 1][dim]: keep every step's pair (else ping-pong)
    // results
    int nstep = 0;
    double norm0 = 0.0;
};

// Widths preset on the jobs from the context's tuning table (the widest
// tuned job decides the block size), or forced (force_* > 0, the tuner).
int preset_widths(edzt_ctx* c, std::vector<LzJob>& jobs, int force_wc, int force_r, int force_block)
{
    if (force_block > 0) {
        for (LzJob& J : jobs) { J.ph[0].width = force_wc; J.ph[1].width = force_r; }
        return force_block;
    }
    int block = 0;
    long long widest = -1;
    for (LzJob& J : jobs) {
        auto it = c->tuned.find({J.S.up.count, J.S.dn.count});
        if (it == c->tuned.end()) continue;
        J.ph[0].width = it->second.wc;
        J.ph[1].width = it->second.r;
        if (J.S.dim > widest) { widest = J.S.dim; block = it->second.block; }
    }
    return block;
}

constexpr size_t kLaunchLog = 256;

void log_launch(edzt_ctx* c, double ms, double bytes, double states)
{
    if (c->log_ms.size() >= kLaunchLog) return;
    c->log_ms.push_back(ms);
    c->log_bytes.push_back(bytes);
    c->log_states.push_back(states);
}

void run_jobs(edzt_ctx* c, std::vector<JobSpec>& specs, int force_wc = 0, int force_r = 0, int force_block = 0)
{
    const int nj = (int)specs.size();
    if (nj == 0) return;
    std::vector<LzJob> jobs(nj);
    std::vector<Lease<double2>> bufs;
    std::vector<Lease<double>> dbufs;
    bufs.reserve((size_t)nj * 2);
    dbufs.reserve((size_t)nj);
    int max_steps = 0;
    for (int j = 0; j < nj; j++) {
        JobSpec& s = specs[j];
        LzJob& J = jobs[j];
        std::memset(&J, 0, sizeof(J));
        J.S = make_sector_mt(c, s.mt ? *s.mt : c->mt, s.nu, s.nd);
        const long long dim = J.S.dim;
        if (s.keep) {
            J.keep = 1;
            J.YW[0] = s.keep;
            J.YW[1] = nullptr;
        } else {
            for (int q = 0; q < 2; q++) {
                bufs.emplace_back(c->pool, (size_t)dim);
                J.YW[q] = bufs.back().p;
            }
        }
        dbufs.emplace_back(c->pool, (size_t)lz_d_size(J.S.up.count, J.S.dn.count));
        J.D = dbufs.back().p;
        J.eig = s.eig;
        J.coeff = s.coeff;
        J.a = s.a;
        J.b = s.b;
        J.maxnstep = s.maxnstep;
        J.mode = s.mode;
        J.init = s.init;
        J.key = s.key;
        J.ac = s.ac;
        J.src = s.ac_src;
        max_steps = std::max(max_steps, J.maxnstep);
        if (s.mode == LZ_COEFF) {
            CK(cudaMemsetAsync(s.a, 0, sizeof(double) * s.maxnstep, c->stream));
            CK(cudaMemsetAsync(s.b, 0, sizeof(double) * s.maxnstep, c->stream));
        }
    }
    // rows per tile and columns per slab of every job (tuned, else by
    // lz_plan's rule), tile lists of both phases, grid and shared memory
    const int prefer = preset_widths(c, jobs, force_wc, force_r, force_block);
    std::vector<long long> prefix;
    const LzPlan P = lz_plan(c->device, jobs.data(), nj, prefix, prefer);
    if (P.grid <= 0) throw EdztError{EDZT_ERR_CUDA, "persistent kernel cannot be resident (shared memory too large)"};
    const int G = P.grid;
    std::vector<LzState> st(2 * (size_t)nj);
    std::memset(st.data(), 0, sizeof(LzState) * st.size());
    for (int j = 0; j < nj; j++) st[2 * (size_t)j + 1].active = 1;   // the state before phase 0 (parity 1)
    const size_t bytes_jobs = sizeof(LzJob) * nj, bytes_st = sizeof(LzState) * st.size();
    const size_t bytes_pre = sizeof(long long) * prefix.size(), bytes_slots = sizeof(double) * 2 * (size_t)P.slots;
    const size_t bytes_sw = lz_sync_bytes(G);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t total = al(bytes_jobs) + al(bytes_st) + al(bytes_pre) + al(bytes_slots) + al(bytes_sw);
    Lease<char> blob(c->pool, total);
    char* base = blob.p;
    LzJob* d_jobs = reinterpret_cast<LzJob*>(base);
    LzState* d_st = reinterpret_cast<LzState*>(base + al(bytes_jobs));
    long long* d_pre = reinterpret_cast<long long*>(base + al(bytes_jobs) + al(bytes_st));
    double* d_slots = reinterpret_cast<double*>(base + al(bytes_jobs) + al(bytes_st) + al(bytes_pre));
    unsigned* d_sw = reinterpret_cast<unsigned*>(base + al(bytes_jobs) + al(bytes_st) + al(bytes_pre) + al(bytes_slots));
    std::vector<unsigned> sw(bytes_sw / sizeof(unsigned), 0u);
    sw[64] = (unsigned)nj;   // runs still going
    for (int j = 0; j < nj; j++) jobs[j].st = d_st + 2 * (size_t)j;
    CK(cudaMemcpyAsync(d_jobs, jobs.data(), bytes_jobs, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_st, st.data(), bytes_st, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_pre, prefix.data(), bytes_pre, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_sw, sw.data(), bytes_sw, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->status->p, 0, sizeof(int), c->stream));
    LzBatch B;
    std::memset(&B, 0, sizeof(B));
    B.njobs = nj;
    B.grid = G;
    B.block = P.block;
    B.smem = P.smem;
    B.total[0] = P.total[0];
    B.total[1] = P.total[1];
    B.max_phases = 2 * max_steps + 4;   // two phases per step and the phase that closes the last one
    if (c->dbg_pass_cap > 0) B.max_phases = std::min(B.max_phases, c->dbg_pass_cap);
    B.wait_ns = c->dbg_wait_ns;
    B.stall_cta = c->dbg_stall_cta;
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(launch_lanczos_persistent(B, d_jobs, d_pre, d_slots, d_sw, c->status->as<int>(), c->stream));
    CK(cudaEventRecord(c->ev1, c->stream));
    c->launches += 1;
    int status = 0;
    CK(cudaMemcpyAsync(st.data(), d_st, bytes_st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&status, c->status->p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (status == EDZT_DEV_BARRIER_TIMEOUT)
        throw EdztError{EDZT_ERR_TIMEOUT, "persistent Lanczos kernel: grid barrier wait timed out"};
    if (status != 0) throw EdztError{EDZT_ERR_CUDA, "persistent Lanczos kernel reported status " + std::to_string(status)};
    double bytes = 0.0;
    for (int j = 0; j < nj; j++) {
        // the final state is the finished one of the two parity copies
        const LzState& s0 = st[2 * (size_t)j];
        const LzState& s1 = st[2 * (size_t)j + 1];
        const LzState* fin = !s0.active ? &s0 : (!s1.active ? &s1 : nullptr);
        if (!fin) throw EdztError{EDZT_ERR_NUMERIC, "Lanczos run did not finish within the pass limit"};
        specs[j].nstep = fin->nstep;
        specs[j].norm0 = fin->norm0;
        const double dim = (double)jobs[j].S.dim;
        const double init = (specs[j].init == LZ_INIT_HASH) ? 8.0 : 16.0;
        const double per_step = (specs[j].mode == LZ_COEFF) ? 24.0 : 40.0;
        bytes += dim * (init + per_step * specs[j].nstep);
    }
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->st_launches += 1;
    c->st_ms += ms;
    c->st_bytes += bytes;
    double states = 0.0;
    for (int j = 0; j < nj; j++) states += (double)jobs[j].S.dim;
    log_launch(c, ms, bytes, states);
}

// ---------------------------------------------------------------------------
// autotuner: the tile shapes of the persistent kernel for one sector shape,
// chosen by timing short runs of every shape that fits: columns per slab WC
// (the column phase's stripe width), rows per tile R, and the CTA shape (two
// CTAs of 256 threads per SM, or one of 512).  The best is recorded on the
// context for the sector's (up strings, down strings) and used by every
// later launch whose budget allows it.
// ---------------------------------------------------------------------------
edzt_ctx::Tuned tune_sector(edzt_ctx* c, int nu, int nd, int steps)
{
    const DevSector S = make_sector(c, nu, nd);
    Lease<double> ab(c->pool, (size_t)2 * steps);
    auto run = [&](int wc, int r, int block) {
        std::vector<JobSpec> specs(1);
        specs[0].nu = nu; specs[0].nd = nd;
        specs[0].mode = LZ_COEFF;
        specs[0].init = LZ_INIT_HASH;
        specs[0].key = edzt_stream_key(0x7475e3ull, 0);
        specs[0].maxnstep = steps;
        specs[0].a = ab.p;
        specs[0].b = ab.p + steps;
        const double ms0 = c->st_ms;
        run_jobs(c, specs, wc, r, block);
        return (c->st_ms - ms0) / std::max(1, specs[0].nstep);
    };
    const size_t fixed = lz_fixed_smem();
    edzt_ctx::Tuned best{0, 0, 0, HUGE_VAL};
    run(2, 1, 512);                                       // warm-up
    for (int block : {256, 512}) {
        const size_t budget = (block == 256 ? 108 * 1024 : kLzSmemMax) - fixed;
        for (int wc : {8, 4, 2}) {
            if (lz_col_smem(S.dn.count, wc) > budget) continue;
            for (int r : {4, 2, 1}) {
                if (lz_row_smem(S.up.count, r) > budget) continue;
                const double ms = run(wc, r, block);
                if (ms < best.ms_per_step) best = {wc, r, block, ms};
            }
        }
    }
    if (best.wc == 0) throw EdztError{EDZT_ERR_ARG, "no tile shape of this sector fits shared memory"};
    c->tuned[{S.up.count, S.dn.count}] = best;
    return best;
}

// ---------------------------------------------------------------------------
// plain engine: the reference's lanczos_iteration step by step, one kernel per
// BLAS-1 operation and a host read of every reduction (src/lanczos_solver.f90)
// ---------------------------------------------------------------------------
double plain_dot(edzt_ctx* c, const double* x, const double* y, long long n)
{
    launch_dot(x, y, n, c->dot_part->as<double>(), c->scal->as<double>(), c->stream);
    c->launches += 2;
    CK(cudaMemcpyAsync(c->pinned, c->scal->p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return c->pinned[0];
}

// lanczos_iteration (lanczos_solver.f90:92-173); a, b host arrays [maxnstep].
int plain_lanczos(edzt_ctx* c, const DevSector& S, const double* v_init, int maxnstep, double* a, double* b,
                  double* norm_out, const double* coeff, double* eig)
{
    const long long n = S.dim;
    Lease<double> v(c->pool, (size_t)n), w(c->pool, (size_t)n),
        hs(c->pool, (size_t)hx_scratch_size(S.up.count, S.dn.count));
    if (coeff == nullptr)
        for (int i = 0; i < maxnstep; i++) { a[i] = 0.0; b[i] = 0.0; }
    const double norm_v = std::sqrt(plain_dot(c, v_init, v_init, n));          // :128
    if (norm_out) *norm_out = norm_v;
    if (!(norm_v > 0.0)) return 0;
    CK(cudaMemcpyAsync(w.p, v_init, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    launch_swap_scale(v.p, w.p, n, nullptr, norm_v, c->stream);                // w = v_init / norm_v :130
    std::swap(v.p, w.p);
    c->launches += 1;
    if (eig) {                                                                 // :254-255
        CK(cudaMemsetAsync(eig, 0, sizeof(double) * n, c->stream));
        launch_axpy(eig, w.p, n, nullptr, coeff[0], 1.0, c->stream);
        c->launches += 1;
    }
    launch_hx(S, w.p, v.p, 0, hs.p, c->stream);                                // :132
    c->launches += 2;
    CKLAUNCH();
    int nstep;
    if (!coeff) a[0] = plain_dot(c, w.p, v.p, n);                              // :134
    if (maxnstep == 1) return 1;                                               // :137-141
    launch_axpy(v.p, w.p, n, nullptr, a[0], -1.0, c->stream);                  // :143
    c->launches += 1;
    if (!coeff) b[1] = std::sqrt(plain_dot(c, v.p, v.p, n));                   // :144
    int k = 2;
    for (;;) {
        if (b[k - 1] < 1.0e-16) { nstep = k - 1; if (!coeff) b[k - 1] = 0.0; break; }
        launch_swap_scale(w.p, v.p, n, nullptr, b[k - 1], c->stream);          // :152-156
        c->launches += 1;
        if (eig) {                                                             // :279
            launch_axpy(eig, w.p, n, nullptr, coeff[k - 1], 1.0, c->stream);
            c->launches += 1;
        }
        launch_hx(S, w.p, v.p, 1, hs.p, c->stream);                            // :158
        c->launches += 2;
        if (!coeff) a[k - 1] = plain_dot(c, w.p, v.p, n);                      // :159
        if (k >= maxnstep) { nstep = k; break; }                               // :161-164
        launch_axpy(v.p, w.p, n, nullptr, a[k - 1], -1.0, c->stream);          // :166
        c->launches += 1;
        if (!coeff) b[k] = std::sqrt(plain_dot(c, v.p, v.p, n));               // :167
        k = k + 1;
    }
    return nstep;
}

// ---------------------------------------------------------------------------
// drivers
// ---------------------------------------------------------------------------
void require_model(edzt_ctx* c)
{
    if (!c->mt.valid) throw EdztError{EDZT_ERR_STATE, "no model: call edzt_set_model first"};
}

void check_sector(edzt_ctx* c, int nu, int nd)
{
    arg_check(sector_valid(c, nu, nd), "electron counts outside [0, nsite]");
}

// Normalise the eigenvector and compute |H g - E g|^2 (lanczos_solver.f90:291-297).
double finish_eigvec(edzt_ctx* c, const DevSector& S, double* vec, double e0)
{
    const long long n = S.dim;
    double* sc = c->scal->as<double>();
    launch_dot(vec, vec, n, c->dot_part->as<double>(), sc, c->stream);
    launch_scale_inv_sqrt(vec, n, sc, c->stream);                              // :291
    Lease<double> v(c->pool, (size_t)n), hs(c->pool, (size_t)hx_scratch_size(S.up.count, S.dn.count));
    launch_hx(S, vec, v.p, 0, hs.p, c->stream);
    launch_axpy(v.p, vec, n, nullptr, e0, -1.0, c->stream);
    c->launches += 7;
    CKLAUNCH();
    return plain_dot(c, v.p, v.p, n);
}

// ---------------------------------------------------------------------------
// diag_arpack (src/arpack_solver.f90:19-124): the lowest eigenpair of a sector
// by a restarted Lanczos with the reference's ARPACK settings: nev = 3 wanted
// eigenvalues, which = 'SA' (smallest algebraic), ncv = 6 basis vectors,
// tol = 0 (machine precision), exact shifts, at most 20000 restarts.
//
// ARPACK's implicit restart with exact shifts keeps the span of the wanted
// Ritz vectors and the residual.  The thick restart (K. Wu and H. Simon,
// SIAM J. Matrix Anal. Appl. 22 (2000) 602-616) keeps that span explicitly:
// the kept Ritz vectors, then the normalised residual, with the projected
// matrix an arrow (Ritz values on the diagonal, beta_m * y_{m,i} on the
// border) that the next Lanczos steps extend.  Convergence is ARPACK's test
// (dsconv): Ritz estimate |beta_m y_{m,i}| <= tol * max(eps^(2/3), |theta_i|)
// for all nev wanted values, tol = eps = 2^-53.  The number kept grows with
// the converged count as in dsaup2: nev + min(nconv, (ncv - nev) / 2).
// Every new vector is orthogonalised against the whole basis twice.
// ---------------------------------------------------------------------------
constexpr int kArNev = 3, kArNcv = 6, kArMaxItr = 20000;

struct ArpackOut {
    double eigval = 0.0;
    double ritz[kArNev] = {0, 0, 0}, bounds[kArNev] = {0, 0, 0}, resid[kArNev] = {0, 0, 0};
    int nmult = 0, nrestart = 0;
};

// vec_out: device [dim], receives the normalised eigenvector of the lowest
// eigenvalue.  with_resid: also the direct residuals |H x_i - theta_i x_i|
// of the nev Ritz vectors (arpack_solver.f90:94-101), three more H.v.
void diag_arpack_impl(edzt_ctx* c, const DevSector& S, uint64_t key, double* vec_out, ArpackOut& R,
                      bool with_resid)
{
    const long long n = S.dim;
    if (n < kArNcv) throw EdztError{EDZT_ERR_ARG, "diag_arpack: sector dimension below ncv = 6"};
    const int m = kArNcv, kmax = kArNev + (kArNcv - kArNev) / 2;
    const double eps = 0x1p-53, eps23 = std::pow(eps, 2.0 / 3.0), tol = eps;
    cudaStream_t st = c->stream;
    Lease<double> buf(c->pool, (size_t)(m + 1 + kmax) * n), hxs(c->pool, (size_t)hx_scratch_size(S.up.count, S.dn.count));
    Lease<double> small(c->pool, (size_t)rl_partials_size() + 32 + EDZT_RL_MAXV * EDZT_RL_MAXV);
    double* part = small.p;
    double* hd = small.p + rl_partials_size();          // [0, 8) pass 1, [8, 16) pass 2, [16] |w|^2
    double* Yd = hd + 32;
    std::vector<double*> spare;
    for (int i = m + 1 + kmax - 1; i >= 0; i--) spare.push_back(buf.p + (size_t)i * n);
    auto take = [&] { double* p = spare.back(); spare.pop_back(); return p; };
    std::vector<double*> V(m + 1, nullptr);
    double T[kArNcv][kArNcv] = {};
    double* hh = c->pinned;                              // 17 host doubles
    // orthogonalise w against V[0..nv) twice; returns |w|^2, projections in hh
    auto orth = [&](double* w, int nv) {
        RlVecs B{};
        for (int q = 0; q < nv; q++) B.p[q] = V[q];
        if (nv > 0) {
            launch_rl_mdot(B, nv, w, n, part, hd, st);
            launch_rl_project_out(w, B, nv, hd, n, st);
            launch_rl_mdot(B, nv, w, n, part, hd + 8, st);
            launch_rl_project_out(w, B, nv, hd + 8, n, st);
            c->launches += 6;
        }
        RlVecs W{};
        W.p[0] = w;
        launch_rl_mdot(W, 1, w, n, part, hd + 16, st);
        c->launches += 2;
        CKLAUNCH();
        CK(cudaMemcpyAsync(hh, hd, sizeof(double) * 17, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return hh[16];
    };
    // a random unit vector orthogonal to V[0..nv) into V[nv]
    auto random_vector = [&](int nv, uint64_t stream_no) {
        for (int tries = 0; tries < 3; tries++) {
            launch_fill_start(V[nv], n, edzt_stream_key(key, stream_no + (uint64_t)tries), st);
            c->launches += 1;
            const double nrm2 = orth(V[nv], nv);
            if (nrm2 > 0.0) {
                launch_rl_div(V[nv], V[nv], std::sqrt(nrm2), n, st);
                c->launches += 1;
                return;
            }
        }
        throw EdztError{EDZT_ERR_NUMERIC, "diag_arpack: no start vector orthogonal to the basis"};
    };
    V[0] = take();
    random_vector(0, 0);
    int k = 0;                                           // basis vectors carried over by the last restart
    double anorm = 0.0, betam = 0.0;
    std::vector<double> theta(m), Y((size_t)m * m);
    for (;;) {
        for (int j = k; j < m; j++) {                    // extend the factorisation to m vectors
            if (!V[j + 1]) V[j + 1] = take();
            double* w = V[j + 1];
            launch_hx(S, V[j], w, 0, hxs.p, st);
            c->launches += 2;
            R.nmult++;
            const double nrm2 = orth(w, j + 1);
            T[j][j] = hh[j] + hh[8 + j];
            const double beta = std::sqrt(std::max(nrm2, 0.0));
            anorm = std::max(anorm, std::fabs(T[j][j]) + beta + (j > 0 ? std::fabs(T[j - 1][j]) : 0.0));
            const bool invariant = !(beta > 1e-13 * anorm);
            if (j + 1 < m) {
                if (invariant) {                          // invariant subspace: restart the recursion
                    random_vector(j + 1, 1000 + (uint64_t)R.nmult);
                    T[j][j + 1] = T[j + 1][j] = 0.0;
                } else {
                    launch_rl_div(w, w, beta, n, st);
                    c->launches += 1;
                    T[j][j + 1] = T[j + 1][j] = beta;
                }
            } else {
                betam = invariant ? 0.0 : beta;
                if (!invariant) {
                    launch_rl_div(w, w, beta, n, st);
                    c->launches += 1;
                }
            }
        }
        double A[kArNcv * kArNcv];
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) A[i * m + j] = T[i][j];
        if (edzt::symmetric_eig(m, A, theta.data(), Y.data()) != 0)
            throw EdztError{EDZT_ERR_NUMERIC, "diag_arpack: non-finite projected matrix"};
        int nconv = 0;
        for (int i = 0; i < kArNev; i++) {
            R.ritz[i] = theta[i];
            R.bounds[i] = std::fabs(betam * Y[(size_t)(m - 1) * m + i]);
            if (R.bounds[i] <= tol * std::max(eps23, std::fabs(theta[i]))) nconv++;
        }
        if (nconv >= kArNev) break;
        if (++R.nrestart > kArMaxItr)
            throw EdztError{EDZT_ERR_NUMERIC, "diag_arpack: not converged in 20000 restarts"};
        // thick restart: V[0..kk) = Ritz vectors, V[kk] = residual, T = arrow
        const int kk = kArNev + std::min(nconv, (kArNcv - kArNev) / 2);
        std::vector<double> Yk((size_t)m * kk);
        for (int j = 0; j < m; j++)
            for (int i = 0; i < kk; i++) Yk[(size_t)j * kk + i] = Y[(size_t)j * m + i];
        CK(cudaMemcpyAsync(Yd, Yk.data(), sizeof(double) * Yk.size(), cudaMemcpyHostToDevice, st));
        RlVecs B{};
        RlOut O{};
        for (int j = 0; j < m; j++) B.p[j] = V[j];
        for (int i = 0; i < kk; i++) O.p[i] = take();
        launch_rl_combine(O, kk, B, m, Yd, n, st);
        c->launches += 1;
        CKLAUNCH();
        CK(cudaStreamSynchronize(st));                   // Yk (pageable) consumed
        double* resid_vec = V[m];
        for (int j = 0; j < m; j++) spare.push_back(V[j]);
        std::fill(V.begin(), V.end(), nullptr);
        for (int i = 0; i < kk; i++) V[i] = O.p[i];
        V[kk] = resid_vec;
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) T[i][j] = 0.0;
        for (int i = 0; i < kk; i++) {
            T[i][i] = theta[i];
            T[i][kk] = T[kk][i] = betam * Y[(size_t)(m - 1) * m + i];
        }
        if (betam == 0.0) random_vector(kk, 2000000 + (uint64_t)R.nrestart);
        k = kk;
    }
    // Ritz vectors (dseupd): the lowest into vec_out, normalised
    const int nvec = with_resid ? kArNev : 1;
    std::vector<double> Yk((size_t)m * nvec);
    for (int j = 0; j < m; j++)
        for (int i = 0; i < nvec; i++) Yk[(size_t)j * nvec + i] = Y[(size_t)j * m + i];
    CK(cudaMemcpyAsync(Yd, Yk.data(), sizeof(double) * Yk.size(), cudaMemcpyHostToDevice, st));
    RlVecs B{};
    RlOut O{};
    for (int j = 0; j < m; j++) B.p[j] = V[j];
    O.p[0] = vec_out;
    for (int i = 1; i < nvec; i++) O.p[i] = take();
    launch_rl_combine(O, nvec, B, m, Yd, n, st);
    c->launches += 1;
    CKLAUNCH();
    for (int i = 0; i < nvec; i++) {
        const double nrm2 = orth(O.p[i], 0);             // |x_i|^2 only
        launch_rl_div(O.p[i], O.p[i], std::sqrt(nrm2), n, st);
        c->launches += 1;
        if (with_resid) {
            double* w = spare.back();
            launch_hx(S, O.p[i], w, 0, hxs.p, st);
            launch_axpy(w, O.p[i], n, nullptr, theta[i], -1.0, st);
            c->launches += 3;
            R.resid[i] = std::sqrt(std::max(orth(w, 0), 0.0));
        }
    }
    R.eigval = theta[0];
}

struct SectorResult {
    int nstep = 0;
    double e = HUGE_VAL;
    std::vector<double> a, b, coeff;
    bool ok = false;
};

// ground_state with diag_solver = 2: diag_arpack on every sector, the lowest
// kept with the same strict rule and tie band as the Lanczos path.
void ground_state_arpack(edzt_ctx* c, int nsector, const int* sectors, uint64_t seed, int* isector, double* e0,
                         double* gsvec, double* e_sector, const uint64_t* streams)
{
    int best = -1;
    double beste = HUGE_VAL;
    for (int i = 0; i < nsector; i++) {
        const int nu = sectors[2 * i], nd = sectors[2 * i + 1];
        if (e_sector) e_sector[i] = NAN;
        const long long dim = sector_dim(c, nu, nd);
        if (dim <= 0) continue;
        DevSector S = make_sector(c, nu, nd);
        Lease<double> vec(c->pool, (size_t)dim);
        ArpackOut R;
        diag_arpack_impl(c, S, edzt_stream_key(seed, streams ? streams[i] : (uint64_t)i), vec.p, R, false);
        if (e_sector) e_sector[i] = R.eigval;
        const double tie = 1.0e-10 * std::max(1.0, std::fabs(beste));
        if (best < 0 || R.eigval < beste - tie) {
            best = i;
            beste = R.eigval;
            c->gs_residual = finish_eigvec(c, S, vec.p, R.eigval);
            c->gs_vec = std::move(vec);
            c->gs_up = nu; c->gs_dn = nd; c->gs_isector = i; c->gs_e0 = R.eigval;
        }
    }
    if (best < 0) throw EdztError{EDZT_ERR_NUMERIC, "no sector produced a ground state"};
    c->has_gs = true;
    *isector = c->gs_isector;
    *e0 = c->gs_e0;
    if (gsvec) copy_out(c, gsvec, c->gs_vec.p, sizeof(double) * sector_dim(c, c->gs_up, c->gs_dn));
    CK(cudaStreamSynchronize(c->stream));
}

// streams (nullable): start-vector stream of each sector; default stream i for sector i.
void ground_state_impl(edzt_ctx* c, int nsector, const int* sectors, int maxnstep, uint64_t seed, int* isector,
                       double* e0, double* gsvec, double* e_sector, const uint64_t* streams = nullptr)
{
    auto stream_of = [&](int i) { return streams ? streams[i] : (uint64_t)i; };
    require_model(c);
    arg_check(nsector >= 1 && sectors != nullptr, "nsector >= 1 and sectors required");
    arg_check(maxnstep >= 1, "maxnstep >= 1");
    for (int i = 0; i < nsector; i++) check_sector(c, sectors[2 * i], sectors[2 * i + 1]);
    c->has_gs = false;
    if (c->diag_solver == EDZT_DIAG_ARPACK) {
        ground_state_arpack(c, nsector, sectors, seed, isector, e0, gsvec, e_sector, streams);
        return;
    }
    std::vector<SectorResult> res(nsector);
    // The scan keeps every step's (y, w) pairs when they fit in half of the
    // device memory that was free when the context was created (queried once:
    // a query per solve can wait on the driver behind other processes'
    // queries): the winner's eigenvector is then one pass over its kept w_k
    // instead of a second run of the recurrence (the same sum, in the same
    // order, of the same vectors).  The pool keeps the blocks for the next solve.
    std::vector<Lease<double2>> kept(nsector);
    bool keep = false;
    if (c->engine == EDZT_ENGINE_FUSED && c->keep_vectors) {
        long long states = 0;
        for (int i = 0; i < nsector; i++) states += std::max(0LL, sector_dim(c, sectors[2 * i], sectors[2 * i + 1]));
        keep = (double)states * (maxnstep + 1) * sizeof(double2) <= 0.5 * (double)c->free_at_create;
    }
    if (c->engine == EDZT_ENGINE_FUSED) {
        std::vector<JobSpec> specs;
        std::vector<int> which;
        Lease<double> ab(c->pool, (size_t)nsector * 2 * maxnstep);
        for (int i = 0; i < nsector; i++) {
            const int nu = sectors[2 * i], nd = sectors[2 * i + 1];
            if (sector_dim(c, nu, nd) <= 0) continue;
            JobSpec s;
            s.nu = nu; s.nd = nd;
            s.mode = LZ_COEFF;
            s.init = LZ_INIT_HASH;
            s.key = edzt_stream_key(seed, stream_of(i));
            s.maxnstep = maxnstep;
            s.a = ab.p + (size_t)(2 * i) * maxnstep;
            s.b = ab.p + (size_t)(2 * i + 1) * maxnstep;
            if (keep) {
                kept[i] = Lease<double2>(c->pool, (size_t)(maxnstep + 1) * sector_dim(c, nu, nd));
                s.keep = kept[i].p;
            }
            specs.push_back(s);
            which.push_back(i);
        }
        run_jobs(c, specs);
        std::vector<double> hab((size_t)nsector * 2 * maxnstep);
        CK(cudaMemcpyAsync(hab.data(), ab.p, sizeof(double) * hab.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (size_t q = 0; q < specs.size(); q++) {
            const int i = which[q];
            SectorResult& r = res[i];
            r.nstep = specs[q].nstep;
            r.a.assign(hab.begin() + (size_t)(2 * i) * maxnstep, hab.begin() + (size_t)(2 * i + 1) * maxnstep);
            r.b.assign(hab.begin() + (size_t)(2 * i + 1) * maxnstep, hab.begin() + (size_t)(2 * i + 2) * maxnstep);
            if (r.nstep >= 1) {
                r.coeff.resize(r.nstep);
                r.ok = edzt::lowest_eigenpair(r.nstep, r.a.data(), r.b.data(), &r.e, r.coeff.data()) == 0;
            }
        }
    }
    // selection (ground_state.f90:62-68), strict with a 1e-10 relative tie band
    int best = -1;
    double beste = HUGE_VAL;
    auto consider = [&](int i) {
        const double tie = 1.0e-10 * std::max(1.0, std::fabs(beste));
        if (best < 0 || res[i].e < beste - tie) { best = i; beste = res[i].e; }
    };
    if (c->engine == EDZT_ENGINE_FUSED) {
        for (int i = 0; i < nsector; i++) {
            if (e_sector) e_sector[i] = res[i].ok ? res[i].e : NAN;
            if (res[i].ok) consider(i);
        }
        if (best < 0) throw EdztError{EDZT_ERR_NUMERIC, "no sector produced a ground state"};
        const int nu = sectors[2 * best], nd = sectors[2 * best + 1];
        const long long dim = sector_dim(c, nu, nd);
        c->gs_vec = Lease<double>(c->pool, (size_t)dim);
        SectorResult& r = res[best];
        Lease<double> cf(c->pool, (size_t)r.nstep), ab(c->pool, (size_t)2 * maxnstep);
        CK(cudaMemcpyAsync(cf.p, r.coeff.data(), sizeof(double) * r.nstep, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(ab.p, r.a.data(), sizeof(double) * maxnstep, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(ab.p + maxnstep, r.b.data(), sizeof(double) * maxnstep, cudaMemcpyHostToDevice, c->stream));
        if (keep) {
            launch_keep_combine(kept[best].p, dim, r.nstep, cf.p, c->gs_vec.p, c->stream);
            c->launches += 1;
            CKLAUNCH();
        } else {
            std::vector<JobSpec> ev(1);
            ev[0].nu = nu; ev[0].nd = nd;
            ev[0].mode = LZ_EIGVEC;
            ev[0].init = LZ_INIT_HASH;
            ev[0].key = edzt_stream_key(seed, stream_of(best));
            ev[0].maxnstep = r.nstep;
            ev[0].coeff = cf.p;
            ev[0].eig = c->gs_vec.p;
            ev[0].a = ab.p;
            ev[0].b = ab.p + maxnstep;
            run_jobs(c, ev);
        }
        for (auto& k : kept) k = Lease<double2>();
        DevSector S = make_sector(c, nu, nd);
        c->gs_residual = finish_eigvec(c, S, c->gs_vec.p, r.e);
        c->gs_up = nu; c->gs_dn = nd; c->gs_isector = best; c->gs_e0 = r.e;
    } else {
        // plain engine: diag_lanczos per sector, eigenvector for every sector
        // as the reference does (ground_state.f90:30-73)
        long long maxdim = 0;
        for (int i = 0; i < nsector; i++) maxdim = std::max(maxdim, sector_dim(c, sectors[2 * i], sectors[2 * i + 1]));
        Lease<double> vin(c->pool, (size_t)maxdim), vec(c->pool, (size_t)maxdim);
        for (int i = 0; i < nsector; i++) {
            const int nu = sectors[2 * i], nd = sectors[2 * i + 1];
            if (e_sector) e_sector[i] = NAN;
            if (sector_dim(c, nu, nd) <= 0) continue;
            DevSector S = make_sector(c, nu, nd);
            launch_fill_start(vin.p, S.dim, edzt_stream_key(seed, stream_of(i)), c->stream);   // :42-46
            c->launches += 1;
            SectorResult& r = res[i];
            r.a.assign(maxnstep, 0.0);
            r.b.assign(maxnstep, 0.0);
            r.nstep = plain_lanczos(c, S, vin.p, maxnstep, r.a.data(), r.b.data(), nullptr, nullptr, nullptr);
            if (r.nstep < 1) continue;
            r.coeff.resize(r.nstep);
            r.ok = edzt::lowest_eigenpair(r.nstep, r.a.data(), r.b.data(), &r.e, r.coeff.data()) == 0;
            if (!r.ok) continue;
            std::vector<double> bb = r.b;
            plain_lanczos(c, S, vin.p, r.nstep, r.a.data(), bb.data(), nullptr, r.coeff.data(), vec.p);
            const double resid = finish_eigvec(c, S, vec.p, r.e);
            if (e_sector) e_sector[i] = r.e;
            const int prev = best;
            consider(i);
            if (best != prev) {
                c->gs_vec = Lease<double>(c->pool, (size_t)S.dim);
                CK(cudaMemcpyAsync(c->gs_vec.p, vec.p, sizeof(double) * S.dim, cudaMemcpyDeviceToDevice, c->stream));
                c->gs_up = nu; c->gs_dn = nd; c->gs_isector = i; c->gs_e0 = r.e; c->gs_residual = resid;
            }
        }
        if (best < 0) throw EdztError{EDZT_ERR_NUMERIC, "no sector produced a ground state"};
    }
    c->has_gs = true;
    *isector = c->gs_isector;
    *e0 = c->gs_e0;
    if (gsvec) copy_out(c, gsvec, c->gs_vec.p, sizeof(double) * sector_dim(c, c->gs_up, c->gs_dn));
    CK(cudaStreamSynchronize(c->stream));
}

// One c^+ or c run of green_diag.
struct GreenRun {
    ModelTables* mt = nullptr;     // model (nullptr: the context's, with its resident ground state)
    const double* gs = nullptr;    // ground state of the run's model (device), sector (gs_up, gs_dn)
    int gs_up = 0, gs_dn = 0;
    double e0 = 0.0;
    const double* start = nullptr; // explicit start vector (device) instead of c^(+)|gs>, e.g. (c_a + c_b)^(+)|gs>
    int iorb, ispin, pm;
    int nu, nd;            // excitation sector
    int nstep = 0;
    double norm0 = 0.0;
    double* a = nullptr;   // device [maxnstep]
    double* b = nullptr;
};

ApplyCArgs applyc_args_ns(edzt_ctx* c, int ns, int in_up, int in_dn, int pm, int iorb, int ispin, int out_up,
                          int out_dn)
{
    ApplyCArgs A{};
    A.pm = pm; A.iorb = iorb; A.ispin = ispin;
    A.nsite = ns;
    StrTable& ou = str_table_ns(c, ns, out_up);
    StrTable& od = str_table_ns(c, ns, out_dn);
    StrTable& iu = str_table_ns(c, ns, in_up);
    StrTable& idn = str_table_ns(c, ns, in_dn);
    A.out_nup = ou.count; A.out_ndn = od.count;
    A.out_up_str = ou.str->as<uint32_t>();
    A.out_dn_str = od.str->as<uint32_t>();
    A.in_nup = iu.count;
    A.in_up_rank = iu.rank->as<int32_t>();
    A.in_dn_rank = idn.rank->as<int32_t>();
    return A;
}

ApplyCArgs applyc_args(edzt_ctx* c, int in_up, int in_dn, int pm, int iorb, int ispin, int out_up, int out_dn)
{
    return applyc_args_ns(c, nsite_of(c), in_up, in_dn, pm, iorb, ispin, out_up, out_dn);
}

void excitation(int nu, int nd, int pm, int ispin, int* ou, int* od)
{
    const int d = (pm == 1) ? 1 : -1;
    *ou = nu + (ispin == 1 ? d : 0);
    *od = nd + (ispin == 2 ? d : 0);
}

// Runs all requested excitation Lanczos runs, then the continued fractions.
// g_out[r]: complex [nw] per run (host), ab_out[r]: host a (maxnstep) + b.
void green_runs(edzt_ctx* c, std::vector<GreenRun>& runs, int maxnstep, int nw, const double* omega_dev,
                std::vector<std::vector<double>>& g_out, std::vector<std::vector<double>>& ab_out,
                int real_axis = 0, double eta = 0.0)
{
    const int nr = (int)runs.size();
    Lease<double> ab(c->pool, (size_t)std::max(nr, 1) * 2 * maxnstep);
    CK(cudaMemsetAsync(ab.p, 0, sizeof(double) * (size_t)std::max(nr, 1) * 2 * maxnstep, c->stream));
    for (int r = 0; r < nr; r++) {
        runs[r].a = ab.p + (size_t)(2 * r) * maxnstep;
        runs[r].b = ab.p + (size_t)(2 * r + 1) * maxnstep;
    }
    for (GreenRun& g : runs)        // runs without a source use the context's resident ground state
        if (!g.mt) { g.mt = &c->mt; g.gs = c->gs_vec.p; g.gs_up = c->gs_up; g.gs_dn = c->gs_dn; g.e0 = c->gs_e0; }
    std::vector<int> live;
    if (c->engine == EDZT_ENGINE_FUSED) {
        std::vector<JobSpec> specs;
        for (int r = 0; r < nr; r++) {
            GreenRun& g = runs[r];
            const int ns = g.mt->model.nsite;
            if (sector_dim_ns(ns, g.nu, g.nd) <= 0) continue;
            JobSpec s;
            s.mt = g.mt;
            s.nu = g.nu; s.nd = g.nd;
            s.mode = LZ_COEFF;
            if (g.start) {
                s.init = LZ_INIT_COPY;
                s.ac_src = g.start;
            } else {
                s.init = LZ_INIT_APPLYC;
                s.ac = applyc_args_ns(c, ns, g.gs_up, g.gs_dn, g.pm, g.iorb, g.ispin, g.nu, g.nd);
                s.ac_src = g.gs;
            }
            s.maxnstep = maxnstep;
            s.a = g.a; s.b = g.b;
            specs.push_back(s);
            live.push_back(r);
        }
        run_jobs(c, specs);
        for (size_t q = 0; q < specs.size(); q++) {
            runs[live[q]].nstep = specs[q].nstep;
            runs[live[q]].norm0 = specs[q].norm0;
        }
    } else {
        for (int r = 0; r < nr; r++) {
            GreenRun& g = runs[r];
            const int ns = g.mt->model.nsite;
            if (sector_dim_ns(ns, g.nu, g.nd) <= 0) continue;
            DevSector S = make_sector_mt(c, *g.mt, g.nu, g.nd);
            Lease<double> vin(c->pool, (size_t)S.dim);
            if (g.start) {
                launch_copy(vin.p, g.start, S.dim, c->stream);
            } else {
                ApplyCArgs A = applyc_args_ns(c, ns, g.gs_up, g.gs_dn, g.pm, g.iorb, g.ispin, g.nu, g.nd);
                launch_apply_c(A, g.gs, vin.p, c->stream);
            }
            c->launches += 1;
            std::vector<double> ha(maxnstep), hb(maxnstep);
            g.nstep = plain_lanczos(c, S, vin.p, maxnstep, ha.data(), hb.data(), &g.norm0, nullptr, nullptr);
            CK(cudaMemcpyAsync(g.a, ha.data(), sizeof(double) * maxnstep, cudaMemcpyHostToDevice, c->stream));
            CK(cudaMemcpyAsync(g.b, hb.data(), sizeof(double) * maxnstep, cudaMemcpyHostToDevice, c->stream));
            CK(cudaStreamSynchronize(c->stream));
        }
    }
    // b(1) = |c^(+)|gs>| (dmft_green.f90:219,249); continued fractions on the device
    Lease<double> g(c->pool, (size_t)std::max(nr, 1) * 2 * nw);
    CK(cudaMemsetAsync(g.p, 0, sizeof(double) * (size_t)std::max(nr, 1) * 2 * nw, c->stream));
    std::vector<CFJob> cj;
    for (int r = 0; r < nr; r++) {
        GreenRun& gr = runs[r];
        if (gr.nstep < 1) continue;
        CFJob J;
        J.a = gr.a; J.b = gr.b;
        J.b1 = gr.norm0;
        // a breakdown after the first vector is evaluated with a zero second level
        J.levels = (gr.nstep == 1 && maxnstep >= 2) ? 2 : gr.nstep;
        J.zr_shift = (gr.pm == 1) ? gr.e0 : -gr.e0;
        J.sign = (gr.pm == 1) ? -1.0 : 1.0;
        J.g = g.p + (size_t)r * 2 * nw;
        cj.push_back(J);
    }
    if (!cj.empty()) {
        Lease<CFJob> dj(c->pool, cj.size());
        CK(cudaMemcpyAsync(dj.p, cj.data(), sizeof(CFJob) * cj.size(), cudaMemcpyHostToDevice, c->stream));
        launch_cf(dj.p, (int)cj.size(), omega_dev, nw, c->stream, real_axis, eta);
        c->launches += 1;
        CKLAUNCH();
        CK(cudaStreamSynchronize(c->stream));
    }
    std::vector<double> hg((size_t)std::max(nr, 1) * 2 * nw), hab((size_t)std::max(nr, 1) * 2 * maxnstep);
    CK(cudaMemcpyAsync(hg.data(), g.p, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hab.data(), ab.p, sizeof(double) * hab.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    g_out.assign(nr, {});
    ab_out.assign(nr, {});
    for (int r = 0; r < nr; r++) {
        g_out[r].assign(hg.begin() + (size_t)r * 2 * nw, hg.begin() + (size_t)(r + 1) * 2 * nw);
        ab_out[r].assign(hab.begin() + (size_t)(2 * r) * maxnstep, hab.begin() + (size_t)(2 * r + 2) * maxnstep);
        if (runs[r].nstep >= 1) ab_out[r][maxnstep] = runs[r].norm0;       // b(1) (:219, :249)
    }
}

void require_gs(edzt_ctx* c)
{
    if (!c->has_gs) throw EdztError{EDZT_ERR_STATE, "no resident ground state: call edzt_ground_state first"};
}

// The c^+ / c runs of cluster_green_ftn (dmft_green.f90:71-100) for a ground
// state in sector (gs_up, gs_dn): per orbital, spin up and (unless even) down.
std::vector<GreenRun> cluster_runs(int norb, bool even, int gs_up, int gs_dn)
{
    std::vector<GreenRun> runs;
    for (int iorb = 1; iorb <= norb; iorb++)
        for (int ispin = 1; ispin <= (even ? 1 : 2); ispin++)
            for (int pm = 1; pm <= 2; pm++) {
                GreenRun g;
                g.iorb = iorb; g.ispin = ispin; g.pm = pm;
                excitation(gs_up, gs_dn, pm, ispin, &g.nu, &g.nd);
                runs.push_back(g);
            }
    return runs;
}

// G_cl(nw, norb, nspin) (complex interleaved) and, nullable, the coefficient
// rows coeffs[norb][2][4][maxnstep] from the results of cluster_runs, which
// start at index r0 of gs / abs_ (dmft_green.f90:102-118).
void assemble_cluster(int norb, int nspin, bool even, int maxnstep, int nw,
                      const std::vector<std::vector<double>>& gs, const std::vector<std::vector<double>>& abs_,
                      size_t r0, double* Gh, double* ch)
{
    size_t r = r0;
    for (int iorb = 1; iorb <= norb; iorb++) {
        std::vector<double> g1(2 * nw, 0.0), g2(2 * nw, 0.0);
        for (int ispin = 1; ispin <= (even ? 1 : 2); ispin++) {
            std::vector<double>& gg = (ispin == 1) ? g1 : g2;
            for (int pm = 1; pm <= 2; pm++, r++) {
                for (int q = 0; q < 2 * nw; q++) gg[q] += gs[r][q];
                if (!ch) continue;
                const double* a = abs_[r].data();
                const double* b = abs_[r].data() + maxnstep;
                double* dst = ch + ((size_t)(iorb - 1) * 2 + (ispin - 1)) * 4 * maxnstep;
                double* da = dst + (pm == 1 ? 0 : 2) * maxnstep;
                double* db = dst + (pm == 1 ? 1 : 3) * maxnstep;
                std::memcpy(da, a, sizeof(double) * maxnstep);
                std::memcpy(db, b, sizeof(double) * maxnstep);
            }
        }
        if (even && ch) {   // spin-down rows repeat spin-up (:102-109)
            double* s1 = ch + ((size_t)(iorb - 1) * 2) * 4 * maxnstep;
            std::memcpy(s1 + 4 * maxnstep, s1, sizeof(double) * 4 * maxnstep);
        }
        for (int iw = 0; iw < nw; iw++) {                                       // :111-118
            const size_t o1 = 2 * ((size_t)iw + (size_t)nw * (iorb - 1));
            const size_t o2 = 2 * ((size_t)iw + (size_t)nw * ((iorb - 1) + (size_t)norb));
            if (nspin == 1 && even) {
                Gh[o1] = g1[2 * iw]; Gh[o1 + 1] = g1[2 * iw + 1];
            } else if (nspin == 1) {
                Gh[o1] = 0.5 * (g1[2 * iw] + g2[2 * iw]);
                Gh[o1 + 1] = 0.5 * (g1[2 * iw + 1] + g2[2 * iw + 1]);
            } else {
                Gh[o1] = g1[2 * iw]; Gh[o1 + 1] = g1[2 * iw + 1];
                Gh[o2] = g2[2 * iw]; Gh[o2 + 1] = g2[2 * iw + 1];
            }
        }
    }
}

// cluster_green_ftn (dmft_green.f90:47-126)
void cluster_green_impl(edzt_ctx* c, int nspin, int maxnstep, int nw, const double* omega, double* G_cl,
                        double* coeffs)
{
    require_model(c);
    require_gs(c);
    arg_check(nspin == 1 || nspin == 2, "nspin must be 1 or 2");
    arg_check(maxnstep >= 1 && nw >= 0, "maxnstep >= 1, nw >= 0");
    const int norb = c->mt.model.norb;
    const bool even = !(nspin == 2 || c->gs_up != c->gs_dn);                    // :76-80
    std::vector<GreenRun> runs = cluster_runs(norb, even, c->gs_up, c->gs_dn);
    InVec om(c, omega, nw);
    std::vector<std::vector<double>> gs, abs_;
    green_runs(c, runs, maxnstep, nw, om.d, gs, abs_);
    std::vector<double> Gh((size_t)2 * nw * norb * nspin, 0.0);
    std::vector<double> ch((size_t)norb * 2 * 4 * maxnstep, 0.0);
    assemble_cluster(norb, nspin, even, maxnstep, nw, gs, abs_, 0, Gh.data(), ch.data());
    if (G_cl) copy_out(c, G_cl, Gh.data(), sizeof(double) * Gh.size());
    if (coeffs) copy_out(c, coeffs, ch.data(), sizeof(double) * ch.size());
    CK(cudaStreamSynchronize(c->stream));
}

void green_diag_impl(edzt_ctx* c, int iorb, int ispin, int maxnstep, int nw, const double* omega, double* ap,
                     double* bp, double* am, double* bm, double* g, int real_axis = 0, double eta = 0.0)
{
    require_model(c);
    require_gs(c);
    arg_check(iorb >= 1 && iorb <= c->mt.model.norb && (ispin == 1 || ispin == 2), "bad iorb/ispin");
    arg_check(maxnstep >= 1 && nw >= 0, "maxnstep >= 1, nw >= 0");
    std::vector<GreenRun> runs(2);
    for (int pm = 1; pm <= 2; pm++) {
        GreenRun& gr = runs[pm - 1];
        gr.iorb = iorb; gr.ispin = ispin; gr.pm = pm;
        excitation(c->gs_up, c->gs_dn, pm, ispin, &gr.nu, &gr.nd);
    }
    InVec om(c, omega, nw);
    std::vector<std::vector<double>> gs, abs_;
    green_runs(c, runs, maxnstep, nw, om.d, gs, abs_, real_axis, eta);
    std::vector<double> gsum(2 * nw, 0.0);
    for (int r = 0; r < 2; r++)
        for (int q = 0; q < 2 * nw; q++) gsum[q] += gs[r][q];
    copy_out(c, ap, abs_[0].data(), sizeof(double) * maxnstep);
    copy_out(c, bp, abs_[0].data() + maxnstep, sizeof(double) * maxnstep);
    copy_out(c, am, abs_[1].data(), sizeof(double) * maxnstep);
    copy_out(c, bm, abs_[1].data() + maxnstep, sizeof(double) * maxnstep);
    copy_out(c, g, gsum.data(), sizeof(double) * 2 * nw);
    CK(cudaStreamSynchronize(c->stream));
}

// The full cluster Green's function matrix G_ab(nw, norb, norb, nspin) on the
// resident ground state.  Beyond the reference, which computes the diagonal
// only (dmft_green.f90:71-121): G_ab = (G_(a+b) - G_aa - G_bb) / 2, where
// G_(a+b) is green_diag's construction for the operator c_a + c_b, i.e. its
// c^+ and c runs start from (c_a^+ + c_b^+)|gs> and (c_a + c_b)|gs>.  The
// diagonal and spin rules are cluster_green_ftn's (:76-80, :111-118).
void cluster_green_matrix_impl(edzt_ctx* c, int nspin, int maxnstep, int nw, const double* omega, double* G)
{
    require_model(c);
    require_gs(c);
    arg_check(nspin == 1 || nspin == 2, "nspin must be 1 or 2");
    arg_check(maxnstep >= 1 && nw >= 0, "maxnstep >= 1, nw >= 0");
    const int norb = c->mt.model.norb, ns = nsite_of(c);
    const bool even = !(nspin == 2 || c->gs_up != c->gs_dn);
    const int nsp = even ? 1 : 2;
    std::vector<GreenRun> runs = cluster_runs(norb, even, c->gs_up, c->gs_dn);   // the diagonal, order (a, spin, pm)
    const size_t ndiag = runs.size();
    std::vector<Lease<double>> starts;
    struct Pair { int a, b, ispin; size_t r; };
    std::vector<Pair> pairs;
    for (int ispin = 1; ispin <= nsp; ispin++)
        for (int a = 1; a <= norb; a++)
            for (int b = a + 1; b <= norb; b++) {
                pairs.push_back({a, b, ispin, runs.size()});
                for (int pm = 1; pm <= 2; pm++) {
                    GreenRun g;
                    g.iorb = a; g.ispin = ispin; g.pm = pm;
                    excitation(c->gs_up, c->gs_dn, pm, ispin, &g.nu, &g.nd);
                    const long long n = sector_dim_ns(ns, g.nu, g.nd);
                    if (n > 0) {     // (c_a + c_b)^(+)|gs> = c_a^(+)|gs> + c_b^(+)|gs>
                        starts.emplace_back(c->pool, (size_t)n);
                        Lease<double> tmp(c->pool, (size_t)n);
                        launch_apply_c(applyc_args(c, c->gs_up, c->gs_dn, pm, a, ispin, g.nu, g.nd), c->gs_vec.p,
                                       starts.back().p, c->stream);
                        launch_apply_c(applyc_args(c, c->gs_up, c->gs_dn, pm, b, ispin, g.nu, g.nd), c->gs_vec.p,
                                       tmp.p, c->stream);
                        launch_axpy(starts.back().p, tmp.p, n, nullptr, 1.0, 1.0, c->stream);
                        c->launches += 3;
                        CK(cudaStreamSynchronize(c->stream));   // tmp goes back to the pool
                        g.start = starts.back().p;
                    }
                    runs.push_back(g);
                }
            }
    CKLAUNCH();
    InVec om(c, omega, nw);
    std::vector<std::vector<double>> gs, abs_;
    green_runs(c, runs, maxnstep, nw, om.d, gs, abs_);
    // g[spin][a][b] per frequency: the diagonal from the single runs, the rest from the pairs
    std::vector<double> gm((size_t)nsp * norb * norb * 2 * nw, 0.0);
    auto at = [&](int sp, int a, int b) { return gm.data() + (((size_t)sp * norb + a) * norb + b) * 2 * nw; };
    size_t r = 0;
    for (int a = 0; a < norb; a++)
        for (int sp = 0; sp < nsp; sp++)
            for (int pm = 1; pm <= 2; pm++, r++)
                for (int q = 0; q < 2 * nw; q++) at(sp, a, a)[q] += gs[r][q];
    (void)ndiag;
    for (const Pair& P : pairs) {
        const int sp = P.ispin - 1, a = P.a - 1, b = P.b - 1;
        for (int q = 0; q < 2 * nw; q++) {
            const double gab = gs[P.r][q] + gs[P.r + 1][q];
            const double v = 0.5 * (gab - at(sp, a, a)[q] - at(sp, b, b)[q]);
            at(sp, a, b)[q] = v;
            at(sp, b, a)[q] = v;
        }
    }
    // G(nw, norb, norb, nspin), column-major, complex interleaved (the spin rule of :111-118)
    std::vector<double> Gh((size_t)2 * nw * norb * norb * nspin, 0.0);
    for (int s = 0; s < nspin; s++)
        for (int b = 0; b < norb; b++)
            for (int a = 0; a < norb; a++)
                for (int iw = 0; iw < nw; iw++) {
                    const size_t o = 2 * ((size_t)iw + (size_t)nw * (a + (size_t)norb * (b + (size_t)norb * s)));
                    double re, im;
                    if (even) {
                        re = at(0, a, b)[2 * iw]; im = at(0, a, b)[2 * iw + 1];
                    } else if (nspin == 1) {
                        re = 0.5 * (at(0, a, b)[2 * iw] + at(1, a, b)[2 * iw]);
                        im = 0.5 * (at(0, a, b)[2 * iw + 1] + at(1, a, b)[2 * iw + 1]);
                    } else {
                        re = at(s, a, b)[2 * iw]; im = at(s, a, b)[2 * iw + 1];
                    }
                    Gh[o] = re; Gh[o + 1] = im;
                }
    copy_out(c, G, Gh.data(), sizeof(double) * Gh.size());
    CK(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// batched solves: many independent impurity instances (each the
// ground_state + cluster_green_ftn pair of src/dmft.f90:76-78), every phase
// of all instances of a wave in one persistent launch
// ---------------------------------------------------------------------------
struct BatchInst {
    DevModel model{};
    std::vector<int> sec;          // [nsector][2]
    int nspin = 1;
    uint64_t seed = 0;
    long long footprint = 0;       // device bytes the instance holds at its peak
    std::unique_ptr<ModelTables> mt;
    int best = -1, gs_up = 0, gs_dn = 0;
    double e0 = 0.0;
    Lease<double> gsvec;
};

template <class F>
void parallel_for(int n, F&& f)
{
    const int nt = std::max(1, std::min(n, (int)std::thread::hardware_concurrency()));
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&] {
            for (int i = next++; i < n; i = next++) f(i);
        });
    for (auto& x : th) x.join();
}

void solve_wave(edzt_ctx* c, std::vector<BatchInst>& B, int i0, int i1, int maxnstep, int nw,
                const double* omega_dev, std::vector<double>& Gall, const std::vector<size_t>& goff)
{
    for (int i = i0; i < i1; i++) {
        B[i].mt = std::make_unique<ModelTables>();
        set_tables_model(*B[i].mt, B[i].model, c->stream);
    }
    // ---- ground-state scan: every sector of every instance (ground_state.f90:28-73)
    struct Owner { int inst, sector; };
    std::vector<JobSpec> specs;
    std::vector<Owner> own;
    for (int i = i0; i < i1; i++) {
        const int ns = B[i].model.nsite;
        for (size_t s = 0; s < B[i].sec.size() / 2; s++) {
            const int nu = B[i].sec[2 * s], nd = B[i].sec[2 * s + 1];
            if (sector_dim_ns(ns, nu, nd) <= 0) continue;
            JobSpec j;
            j.mt = B[i].mt.get();
            j.nu = nu; j.nd = nd;
            j.mode = LZ_COEFF;
            j.init = LZ_INIT_HASH;
            j.key = edzt_stream_key(B[i].seed, (uint64_t)s);
            j.maxnstep = maxnstep;
            specs.push_back(j);
            own.push_back({i, (int)s});
        }
    }
    const int nj = (int)specs.size();
    Lease<double> ab(c->pool, (size_t)std::max(nj, 1) * 2 * maxnstep);
    for (int q = 0; q < nj; q++) {
        specs[q].a = ab.p + (size_t)(2 * q) * maxnstep;
        specs[q].b = ab.p + (size_t)(2 * q + 1) * maxnstep;
    }
    run_jobs(c, specs);
    std::vector<double> hab((size_t)std::max(nj, 1) * 2 * maxnstep);
    CK(cudaMemcpyAsync(hab.data(), ab.p, sizeof(double) * hab.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<SectorResult> res(nj);
    parallel_for(nj, [&](int q) {
        SectorResult& r = res[q];
        r.nstep = specs[q].nstep;
        if (r.nstep < 1) return;
        r.coeff.resize(r.nstep);
        r.ok = edzt::lowest_eigenpair(r.nstep, hab.data() + (size_t)(2 * q) * maxnstep,
                                      hab.data() + (size_t)(2 * q + 1) * maxnstep, &r.e, r.coeff.data()) == 0;
    });
    // selection per instance in sector order, 1e-10 relative tie band (ground_state.f90:62-68)
    std::vector<int> win(B.size(), -1);
    for (int q = 0; q < nj; q++) {
        if (!res[q].ok) continue;
        const int i = own[q].inst;
        const int w = win[i];
        const double tie = 1.0e-10 * std::max(1.0, std::fabs(w < 0 ? 0.0 : res[w].e));
        if (w < 0 || res[q].e < res[w].e - tie) win[i] = q;
    }
    // ---- eigenvector pass of every winner (lanczos_solver.f90:213-300)
    std::vector<JobSpec> ev;
    Lease<double> coeffs(c->pool, (size_t)std::max(i1 - i0, 1) * maxnstep);
    std::vector<double> hcoef((size_t)std::max(i1 - i0, 1) * maxnstep, 0.0);
    for (int i = i0; i < i1; i++) {
        const int q = win[i];
        if (q < 0) throw EdztError{EDZT_ERR_NUMERIC, "instance " + std::to_string(i) + ": no sector produced a ground state"};
        BatchInst& I = B[i];
        I.best = own[q].sector;
        I.gs_up = specs[q].nu; I.gs_dn = specs[q].nd;
        I.e0 = res[q].e;
        I.gsvec = Lease<double>(c->pool, (size_t)sector_dim_ns(I.model.nsite, I.gs_up, I.gs_dn));
        std::copy(res[q].coeff.begin(), res[q].coeff.end(), hcoef.begin() + (size_t)(i - i0) * maxnstep);
        JobSpec j;
        j.mt = I.mt.get();
        j.nu = I.gs_up; j.nd = I.gs_dn;
        j.mode = LZ_EIGVEC;
        j.init = LZ_INIT_HASH;
        j.key = specs[q].key;
        j.maxnstep = res[q].nstep;
        j.coeff = coeffs.p + (size_t)(i - i0) * maxnstep;
        j.eig = I.gsvec.p;
        j.a = specs[q].a;            // the coefficients of the scan, still on the device
        j.b = specs[q].b;
        ev.push_back(j);
    }
    CK(cudaMemcpyAsync(coeffs.p, hcoef.data(), sizeof(double) * hcoef.size(), cudaMemcpyHostToDevice, c->stream));
    run_jobs(c, ev);
    for (int i = i0; i < i1; i++) {   // normalise (lanczos_solver.f90:291)
        const long long n = sector_dim_ns(B[i].model.nsite, B[i].gs_up, B[i].gs_dn);
        launch_dot(B[i].gsvec.p, B[i].gsvec.p, n, c->dot_part->as<double>(), c->scal->as<double>(), c->stream);
        launch_scale_inv_sqrt(B[i].gsvec.p, n, c->scal->as<double>(), c->stream);
        c->launches += 3;
    }
    CKLAUNCH();
    // ---- Green's function runs of every instance (dmft_green.f90:47-126)
    std::vector<GreenRun> runs;
    std::vector<size_t> r0(B.size(), 0);
    for (int i = i0; i < i1; i++) {
        BatchInst& I = B[i];
        const bool even = !(I.nspin == 2 || I.gs_up != I.gs_dn);
        r0[i] = runs.size();
        for (GreenRun g : cluster_runs(I.model.norb, even, I.gs_up, I.gs_dn)) {
            g.mt = I.mt.get();
            g.gs = I.gsvec.p;
            g.gs_up = I.gs_up; g.gs_dn = I.gs_dn;
            g.e0 = I.e0;
            runs.push_back(g);
        }
    }
    std::vector<std::vector<double>> gs, abs_;
    green_runs(c, runs, maxnstep, nw, omega_dev, gs, abs_);
    for (int i = i0; i < i1; i++) {
        BatchInst& I = B[i];
        const bool even = !(I.nspin == 2 || I.gs_up != I.gs_dn);
        assemble_cluster(I.model.norb, I.nspin, even, maxnstep, nw, gs, abs_, r0[i], Gall.data() + goff[i], nullptr);
        I.gsvec.reset();
        I.mt.reset();
    }
}

// Validate one instance and estimate the device memory it holds at its peak
// (sector scan: 32 B per state of every sector; Green's runs: 4*norb runs of
// the largest neighbouring sector plus the ground state).
void init_inst(const edzt_instance& in, BatchInst& I)
{
    I.model = model_from(in.norb, in.nbath, in.em, in.ek, in.vmk, in.U, in.Up, in.Jex, in.Jp, in.mu);
    arg_check(in.nsector >= 1 && in.sectors != nullptr, "every instance needs nsector >= 1 sectors");
    arg_check(in.nspin == 1 || in.nspin == 2, "nspin must be 1 or 2");
    I.sec.assign(in.sectors, in.sectors + 2 * in.nsector);
    I.nspin = in.nspin;
    I.seed = in.seed;
    const int ns = I.model.nsite;
    long long gsb = 0, maxd = 0, maxe = 0;
    for (int s = 0; s < in.nsector; s++) {
        const int nu = I.sec[2 * s], nd = I.sec[2 * s + 1];
        arg_check(sector_valid_ns(ns, nu, nd), "electron counts outside [0, nsite]");
        const long long d = sector_dim_ns(ns, nu, nd);
        gsb += 40 * d + 56 * sector_dim_ns(ns, 0, nd);   // two pair buffers and D (slab padding) per run
        maxd = std::max(maxd, d);
        for (int du = -1; du <= 1; du++)
            for (int dd = -1; dd <= 1; dd++)
                if ((du == 0) != (dd == 0)) maxe = std::max(maxe, sector_dim_ns(ns, nu + du, nd + dd));
    }
    const long long cfb = 4LL * I.model.norb * (40 * maxe + 56 * sector_dim_ns(ns, 0, ns / 2)) + 8 * maxd;
    I.footprint = std::max(gsb, cfb) + 56 * maxd;
}

void solve_batch_impl(edzt_ctx* c, int ninst, const edzt_instance* inst, int maxnstep, int nw, const double* omega,
                      int* isector, double* e0, double* G_cl, size_t budget)
{
    arg_check(ninst >= 0 && (ninst == 0 || inst != nullptr), "ninst >= 0 and inst required");
    arg_check(maxnstep >= 1 && nw >= 0 && (nw == 0 || omega != nullptr), "maxnstep >= 1, nw >= 0, omega");
    std::vector<BatchInst> B(ninst);
    std::vector<size_t> goff(ninst + 1, 0);
    for (int i = 0; i < ninst; i++) {
        init_inst(inst[i], B[i]);
        goff[i + 1] = goff[i] + (size_t)2 * nw * B[i].model.norb * B[i].nspin;
    }
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        budget = fr / 10 * 8;
    }
    InVec om(c, omega, nw);
    std::vector<double> Gall(std::max(goff[ninst], (size_t)1), 0.0);
    for (int i0 = 0; i0 < ninst;) {   // waves that fit the device-memory budget
        int i1 = i0;
        long long sum = 0;
        while (i1 < ninst && (i1 == i0 || sum + B[i1].footprint <= (long long)budget)) sum += B[i1++].footprint;
        solve_wave(c, B, i0, i1, maxnstep, nw, om.d, Gall, goff);
        c->pool.trim();
        i0 = i1;
    }
    for (int i = 0; i < ninst; i++) {
        if (isector) isector[i] = B[i].best;
        if (e0) e0[i] = B[i].e0;
    }
    if (G_cl && goff[ninst] > 0) copy_out(c, G_cl, Gall.data(), sizeof(double) * goff[ninst]);
    CK(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// served form: continuous batching of impurity solves at the granularity of
// Lanczos phases.  A request goes through three phases (sector scan,
// eigenvector pass, c / c^+ runs with the continued fractions); the Lanczos
// runs of a phase are live jobs whose buffers and recurrence state persist
// across launches.  Every step serves one size class of requests (classes
// by nsite, the small ones together, taken in turn): it runs slices of that
// class's live runs (persistent launches of a budget of phases, ending with
// every unfinished run's next step opened, so a later launch resumes it)
// and moves requests on as their phase's runs finish, until the step's time
// budget is spent or the class has nothing left to run.  Requests queued
// meanwhile are admitted at the next step when their device-memory
// footprint fits; a small request is thus never held behind the scans of
// large ones for longer than their steps' time budgets.
// ---------------------------------------------------------------------------
struct LiveJob {
    JobSpec spec;
    DevSector S{};
    Lease<double2> yw0, yw1;
    Lease<double> d;
    Lease<LzState> st;                     // [2] by phase parity, on the device
    int k = 0;                             // steps done (host view, from the last slice)
    bool done = false;
};

struct ServReq {
    long long id = 0;
    BatchInst I;
    int phase = 0;                         // 1 scan, 2 eigenvector, 3 Green's runs, 4 done
    int cls = 0;                           // size class
    bool cancelled = false;
    Lease<double> ab;                      // [nsector][2][maxnstep] scan coefficients (device)
    std::vector<int> job_of_sector;        // live scan job of each sector, -1 if none
    std::vector<double> hab;               // scan coefficients on the host
    std::vector<SectorResult> res;
    int win = -1;                          // winning sector
    Lease<double> coef;                    // tridiagonal eigenvector of the winner (device)
    std::vector<GreenRun> runs;
    Lease<double> gab;                     // [nruns][2][maxnstep] Green's-run coefficients (device)
    std::vector<double> G;                 // G_cl(nw, norb, nspin), complex interleaved
    std::vector<std::unique_ptr<LiveJob>> jobs;   // the live runs of the current phase
    std::string error;
};

}  // namespace

struct edzt_server {
    edzt_ctx* c = nullptr;
    int maxnstep = 0, nw = 0;
    std::unique_ptr<DevBuf> omega;
    long long budget = 0, reserved = 0, next_id = 1;
    double step_ms = 25.0;                 // time budget of one step
    int last_cls = -1;                     // class served by the last step
    std::map<int, double> ms_per_phase;    // measured phase time by class
    std::deque<std::unique_ptr<ServReq>> queue;
    std::vector<std::unique_ptr<ServReq>> active;
    std::map<long long, std::unique_ptr<ServReq>> finished;
};

namespace {

// Size class of a request: its nsite, the requests up to nsite 11 together.
int size_class(const BatchInst& I) { return std::max(I.model.nsite, 11); }

std::unique_ptr<LiveJob> make_live(edzt_ctx* c, const JobSpec& spec)
{
    auto L = std::make_unique<LiveJob>();
    L->spec = spec;
    L->S = make_sector_mt(c, spec.mt ? *spec.mt : c->mt, spec.nu, spec.nd);
    L->yw0 = Lease<double2>(c->pool, (size_t)L->S.dim);
    L->yw1 = Lease<double2>(c->pool, (size_t)L->S.dim);
    L->d = Lease<double>(c->pool, (size_t)lz_d_size(L->S.up.count, L->S.dn.count));
    L->st = Lease<LzState>(c->pool, 2);
    LzState init[2];
    std::memset(init, 0, sizeof(init));
    init[1].active = 1;                                  // the state before the first phase (parity 1)
    CK(cudaMemcpyAsync(L->st.p, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));                // init (host memory) consumed
    if (spec.mode == LZ_COEFF) {
        CK(cudaMemsetAsync(spec.a, 0, sizeof(double) * spec.maxnstep, c->stream));
        CK(cudaMemsetAsync(spec.b, 0, sizeof(double) * spec.maxnstep, c->stream));
    }
    return L;
}

// One slice: at most `phases` phases (even) of every live run in v, in one
// persistent launch; runs that finish are marked done with nstep and norm0.
// Returns the launch's device time in ms.
float run_slice(edzt_ctx* c, std::vector<LiveJob*>& v, int phases)
{
    const int nj = (int)v.size();
    std::vector<LzJob> jobs(nj);
    for (int j = 0; j < nj; j++) {
        LiveJob& L = *v[j];
        LzJob& J = jobs[j];
        std::memset(&J, 0, sizeof(J));
        J.S = L.S;
        J.YW[0] = L.yw0.p;
        J.YW[1] = L.yw1.p;
        J.D = L.d.p;
        J.eig = L.spec.eig;
        J.coeff = L.spec.coeff;
        J.a = L.spec.a;
        J.b = L.spec.b;
        J.maxnstep = L.spec.maxnstep;
        J.mode = L.spec.mode;
        J.init = L.spec.init;
        J.key = L.spec.key;
        J.ac = L.spec.ac;
        J.src = L.spec.ac_src;
        J.st = L.st.p;
    }
    const int prefer = preset_widths(c, jobs, 0, 0, 0);
    std::vector<long long> prefix;
    const LzPlan P = lz_plan(c->device, jobs.data(), nj, prefix, prefer);
    if (P.grid <= 0) throw EdztError{EDZT_ERR_CUDA, "persistent kernel cannot be resident (shared memory too large)"};
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t bytes_jobs = sizeof(LzJob) * nj, bytes_pre = sizeof(long long) * prefix.size();
    const size_t bytes_slots = sizeof(double) * 2 * (size_t)P.slots, bytes_sw = lz_sync_bytes(P.grid);
    Lease<char> blob(c->pool, al(bytes_jobs) + al(bytes_pre) + al(bytes_slots) + al(bytes_sw));
    LzJob* d_jobs = reinterpret_cast<LzJob*>(blob.p);
    long long* d_pre = reinterpret_cast<long long*>(blob.p + al(bytes_jobs));
    double* d_slots = reinterpret_cast<double*>(blob.p + al(bytes_jobs) + al(bytes_pre));
    unsigned* d_sw = reinterpret_cast<unsigned*>(blob.p + al(bytes_jobs) + al(bytes_pre) + al(bytes_slots));
    std::vector<unsigned> sw(bytes_sw / sizeof(unsigned), 0u);
    sw[64] = (unsigned)nj;
    CK(cudaMemcpyAsync(d_jobs, jobs.data(), bytes_jobs, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_pre, prefix.data(), bytes_pre, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_sw, sw.data(), bytes_sw, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->status->p, 0, sizeof(int), c->stream));
    LzBatch B;
    std::memset(&B, 0, sizeof(B));
    B.njobs = nj;
    B.grid = P.grid;
    B.block = P.block;
    B.smem = P.smem;
    B.total[0] = P.total[0];
    B.total[1] = P.total[1];
    B.max_phases = std::max(2, phases & ~1);
    if (c->dbg_pass_cap > 0) B.max_phases = std::min(B.max_phases, std::max(2, c->dbg_pass_cap & ~1));
    B.wait_ns = c->dbg_wait_ns;
    B.stall_cta = c->dbg_stall_cta;
    B.slice = 1;
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(launch_lanczos_persistent(B, d_jobs, d_pre, d_slots, d_sw, c->status->as<int>(), c->stream));
    CK(cudaEventRecord(c->ev1, c->stream));
    c->launches += 1;
    std::vector<LzState> st(2 * (size_t)nj);
    for (int j = 0; j < nj; j++)
        CK(cudaMemcpyAsync(&st[2 * (size_t)j], v[j]->st.p, 2 * sizeof(LzState), cudaMemcpyDeviceToHost, c->stream));
    int status = 0;
    CK(cudaMemcpyAsync(&status, c->status->p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (status == EDZT_DEV_BARRIER_TIMEOUT)
        throw EdztError{EDZT_ERR_TIMEOUT, "persistent Lanczos kernel: grid barrier wait timed out"};
    if (status != 0) throw EdztError{EDZT_ERR_CUDA, "persistent Lanczos kernel reported status " + std::to_string(status)};
    double bytes = 0.0;
    for (int j = 0; j < nj; j++) {
        LiveJob& L = *v[j];
        const LzState& s0 = st[2 * (size_t)j];
        const LzState& s1 = st[2 * (size_t)j + 1];
        const LzState* fin = !s0.active ? &s0 : (!s1.active ? &s1 : nullptr);
        const int k_now = fin ? fin->nstep : std::max(s0.k, s1.k) - 1;   // an opened step is not done yet
        const double per_step = (L.spec.mode == LZ_COEFF) ? 24.0 : 40.0;
        if (L.k == 0 && k_now > 0) bytes += (double)L.S.dim * ((L.spec.init == LZ_INIT_HASH) ? 8.0 : 16.0);
        bytes += (double)L.S.dim * per_step * std::max(0, k_now - L.k);
        L.k = std::max(L.k, k_now);
        if (fin) {
            L.done = true;
            L.spec.nstep = fin->nstep;
            L.spec.norm0 = fin->norm0;
        }
    }
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->st_launches += 1;
    c->st_ms += ms;
    c->st_bytes += bytes;
    double states = 0.0;
    for (int j = 0; j < nj; j++) states += (double)jobs[j].S.dim;
    log_launch(c, ms, bytes, states);
    return ms;
}

void server_admit(edzt_server* sv)
{
    edzt_ctx* c = sv->c;
    while (!sv->queue.empty()) {
        ServReq& q = *sv->queue.front();
        if (!sv->active.empty() && sv->reserved + q.I.footprint > sv->budget) break;
        sv->reserved += q.I.footprint;
        q.I.mt = std::make_unique<ModelTables>();
        set_tables_model(*q.I.mt, q.I.model, c->stream);
        const int ns = (int)q.I.sec.size() / 2;
        q.ab = Lease<double>(c->pool, (size_t)std::max(ns, 1) * 2 * sv->maxnstep);
        q.cls = size_class(q.I);
        q.phase = 1;
        // the scan: one run per sector (ground_state.f90:28-73)
        const int nsite = q.I.model.nsite;
        q.job_of_sector.assign(ns, -1);
        for (int s = 0; s < ns; s++) {
            const int nu = q.I.sec[2 * s], nd = q.I.sec[2 * s + 1];
            if (sector_dim_ns(nsite, nu, nd) <= 0) continue;
            JobSpec j;
            j.mt = q.I.mt.get();
            j.nu = nu; j.nd = nd;
            j.mode = LZ_COEFF;
            j.init = LZ_INIT_HASH;
            j.key = edzt_stream_key(q.I.seed, (uint64_t)s);
            j.maxnstep = sv->maxnstep;
            j.a = q.ab.p + (size_t)(2 * s) * sv->maxnstep;
            j.b = q.ab.p + (size_t)(2 * s + 1) * sv->maxnstep;
            q.job_of_sector[s] = (int)q.jobs.size();
            q.jobs.push_back(make_live(c, j));
        }
        sv->active.push_back(std::move(sv->queue.front()));
        sv->queue.pop_front();
    }
}

bool phase_done(const ServReq& q)
{
    for (const auto& j : q.jobs)
        if (!j->done) return false;
    return true;
}

// Scan finished: the tridiagonal ground state of every sector, the winner
// (ground_state.f90:62-68, 1e-10 tie band) and its eigenvector pass.
void after_scan(edzt_server* sv, ServReq& q)
{
    edzt_ctx* c = sv->c;
    const int maxnstep = sv->maxnstep;
    const int nsec = (int)q.I.sec.size() / 2;
    q.hab.assign((size_t)std::max(nsec, 1) * 2 * maxnstep, 0.0);
    CK(cudaMemcpyAsync(q.hab.data(), q.ab.p, sizeof(double) * q.hab.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    q.res.assign(nsec, SectorResult{});
    for (int s = 0; s < nsec; s++) {
        const int jq = q.job_of_sector[s];
        if (jq < 0) continue;
        SectorResult& r = q.res[s];
        r.nstep = q.jobs[jq]->spec.nstep;
        if (r.nstep < 1) continue;
        r.coeff.resize(r.nstep);
        r.ok = edzt::lowest_eigenpair(r.nstep, q.hab.data() + (size_t)(2 * s) * maxnstep,
                                      q.hab.data() + (size_t)(2 * s + 1) * maxnstep, &r.e, r.coeff.data()) == 0;
    }
    int w = -1;
    for (int s = 0; s < nsec; s++) {
        if (!q.res[s].ok) continue;
        const double tie = 1.0e-10 * std::max(1.0, std::fabs(w < 0 ? 0.0 : q.res[w].e));
        if (w < 0 || q.res[s].e < q.res[w].e - tie) w = s;
    }
    q.jobs.clear();
    if (w < 0) { q.error = "no sector produced a ground state"; q.phase = 4; return; }
    q.win = w;
    q.I.best = w;
    q.I.gs_up = q.I.sec[2 * w]; q.I.gs_dn = q.I.sec[2 * w + 1];
    q.I.e0 = q.res[w].e;
    q.I.gsvec = Lease<double>(c->pool, (size_t)sector_dim_ns(q.I.model.nsite, q.I.gs_up, q.I.gs_dn));
    q.coef = Lease<double>(c->pool, (size_t)q.res[w].nstep);
    CK(cudaMemcpyAsync(q.coef.p, q.res[w].coeff.data(), sizeof(double) * q.res[w].nstep, cudaMemcpyHostToDevice,
                       c->stream));
    JobSpec j;                                            // eigenvector pass (lanczos_solver.f90:213-300)
    j.mt = q.I.mt.get();
    j.nu = q.I.gs_up; j.nd = q.I.gs_dn;
    j.mode = LZ_EIGVEC;
    j.init = LZ_INIT_HASH;
    j.key = edzt_stream_key(q.I.seed, (uint64_t)w);
    j.maxnstep = q.res[w].nstep;
    j.coeff = q.coef.p;
    j.eig = q.I.gsvec.p;
    j.a = q.ab.p + (size_t)(2 * w) * maxnstep;
    j.b = q.ab.p + (size_t)(2 * w + 1) * maxnstep;
    q.jobs.push_back(make_live(c, j));
    q.phase = 2;
}

// Eigenvector pass finished: normalise it (lanczos_solver.f90:291) and start
// the c / c^+ runs (dmft_green.f90:204-250).
void after_eigvec(edzt_server* sv, ServReq& q)
{
    edzt_ctx* c = sv->c;
    const int maxnstep = sv->maxnstep;
    BatchInst& I = q.I;
    const long long n = sector_dim_ns(I.model.nsite, I.gs_up, I.gs_dn);
    launch_dot(I.gsvec.p, I.gsvec.p, n, c->dot_part->as<double>(), c->scal->as<double>(), c->stream);
    launch_scale_inv_sqrt(I.gsvec.p, n, c->scal->as<double>(), c->stream);
    c->launches += 3;
    CKLAUNCH();
    const bool even = !(I.nspin == 2 || I.gs_up != I.gs_dn);
    q.runs = cluster_runs(I.model.norb, even, I.gs_up, I.gs_dn);
    q.gab = Lease<double>(c->pool, std::max<size_t>(q.runs.size(), 1) * 2 * maxnstep);
    CK(cudaMemsetAsync(q.gab.p, 0, sizeof(double) * std::max<size_t>(q.runs.size(), 1) * 2 * maxnstep, c->stream));
    q.jobs.clear();
    const int ns = I.model.nsite;
    for (size_t r = 0; r < q.runs.size(); r++) {
        GreenRun& g = q.runs[r];
        g.mt = I.mt.get();
        g.gs = I.gsvec.p;
        g.gs_up = I.gs_up; g.gs_dn = I.gs_dn;
        g.e0 = I.e0;
        g.a = q.gab.p + (2 * r) * maxnstep;
        g.b = q.gab.p + (2 * r + 1) * maxnstep;
        g.nstep = 0;
        if (sector_dim_ns(ns, g.nu, g.nd) <= 0) continue;
        JobSpec j;
        j.mt = I.mt.get();
        j.nu = g.nu; j.nd = g.nd;
        j.mode = LZ_COEFF;
        j.init = LZ_INIT_APPLYC;
        j.ac = applyc_args_ns(c, ns, g.gs_up, g.gs_dn, g.pm, g.iorb, g.ispin, g.nu, g.nd);
        j.ac_src = g.gs;
        j.maxnstep = maxnstep;
        j.a = g.a; j.b = g.b;
        g.nstep = -1 - (int)q.jobs.size();              // its live run, resolved when it finishes
        q.jobs.push_back(make_live(c, j));
    }
    q.phase = 3;
}

// Green's runs finished: continued fractions and G_cl.
void after_green(edzt_server* sv, ServReq& q)
{
    edzt_ctx* c = sv->c;
    const int maxnstep = sv->maxnstep, nw = sv->nw;
    BatchInst& I = q.I;
    std::vector<CFJob> cj;
    const size_t ng = q.runs.size();
    Lease<double> g(c->pool, std::max<size_t>(ng, 1) * 2 * nw);
    CK(cudaMemsetAsync(g.p, 0, sizeof(double) * std::max<size_t>(ng, 1) * 2 * nw, c->stream));
    for (size_t r = 0; r < ng; r++) {
        GreenRun& gr = q.runs[r];
        if (gr.nstep < 0) {
            const LiveJob& L = *q.jobs[-1 - gr.nstep];
            gr.nstep = L.spec.nstep;
            gr.norm0 = L.spec.norm0;
        }
        if (gr.nstep < 1) continue;
        CFJob J;
        J.a = gr.a; J.b = gr.b;
        J.b1 = gr.norm0;
        J.levels = (gr.nstep == 1 && maxnstep >= 2) ? 2 : gr.nstep;
        J.zr_shift = (gr.pm == 1) ? gr.e0 : -gr.e0;
        J.sign = (gr.pm == 1) ? -1.0 : 1.0;
        J.g = g.p + r * 2 * nw;
        cj.push_back(J);
    }
    if (!cj.empty()) {
        Lease<CFJob> dj(c->pool, cj.size());
        CK(cudaMemcpyAsync(dj.p, cj.data(), sizeof(CFJob) * cj.size(), cudaMemcpyHostToDevice, c->stream));
        launch_cf(dj.p, (int)cj.size(), sv->omega->as<double>(), nw, c->stream);
        c->launches += 1;
        CKLAUNCH();
        CK(cudaStreamSynchronize(c->stream));              // dj and its CF jobs consumed
    }
    std::vector<double> hg(std::max<size_t>(ng, 1) * 2 * nw);
    CK(cudaMemcpyAsync(hg.data(), g.p, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<std::vector<double>> gs(ng), abs_(ng);
    for (size_t r = 0; r < ng; r++) gs[r].assign(hg.begin() + r * 2 * nw, hg.begin() + (r + 1) * 2 * nw);
    const bool even = !(I.nspin == 2 || I.gs_up != I.gs_dn);
    q.G.assign((size_t)2 * nw * I.model.norb * I.nspin, 0.0);
    assemble_cluster(I.model.norb, I.nspin, even, maxnstep, nw, gs, abs_, 0, q.G.data(), nullptr);
    q.jobs.clear();
    q.phase = 4;
}

// One step: admit what fits, then serve the next size class in turn.
int server_step(edzt_server* sv)
{
    edzt_ctx* c = sv->c;
    server_admit(sv);
    for (auto& up : sv->active)                               // cancelled requests leave now
        if (up->cancelled) { up->error = "cancelled"; up->jobs.clear(); up->phase = 4; }
    std::vector<int> classes;
    for (auto& up : sv->active)
        if (up->phase < 4) classes.push_back(up->cls);
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    if (!classes.empty()) {
        auto it = std::upper_bound(classes.begin(), classes.end(), sv->last_cls);
        const int cls = (it == classes.end()) ? classes.front() : *it;
        sv->last_cls = cls;
        double left = sv->step_ms;
        for (int round = 0; round < 64; round++) {
            std::vector<LiveJob*> v;
            long long dims = 0;
            for (auto& up : sv->active) {
                if (up->cls != cls || up->phase >= 4) continue;
                for (auto& j : up->jobs)
                    if (!j->done) { v.push_back(j.get()); dims += j->S.dim; }
            }
            if (v.empty()) break;
            auto est = sv->ms_per_phase.find(cls);
            const double mpp = (est != sv->ms_per_phase.end()) ? est->second : 0.01 + (double)dims * 40.0 / 4.0e9;
            int phases = (int)std::min(4096.0, std::max(2.0, left / std::max(mpp, 1e-4)));
            phases &= ~1;
            if (phases < 2) phases = 2;
            const float ms = run_slice(c, v, phases);
            const double per = ms / phases;
            sv->ms_per_phase[cls] = (est != sv->ms_per_phase.end()) ? 0.5 * (est->second + per) : per;
            left -= ms;
            for (auto& up : sv->active) {                     // requests move on as their phase's runs finish
                if (up->cls != cls || up->phase >= 4 || !phase_done(*up)) continue;
                if (up->phase == 1) after_scan(sv, *up);
                else if (up->phase == 2) after_eigvec(sv, *up);
                else if (up->phase == 3) after_green(sv, *up);
            }
            if (left <= 0.0) break;
        }
    }
    CK(cudaStreamSynchronize(c->stream));
    int nfin = 0;                                             // retire finished requests, free their memory
    for (auto it = sv->active.begin(); it != sv->active.end();) {
        if ((*it)->phase == 4) {
            ServReq& q = **it;
            q.jobs.clear();
            q.I.gsvec.reset(); q.I.mt.reset(); q.ab.reset(); q.coef.reset(); q.gab.reset();
            sv->reserved -= q.I.footprint;
            sv->finished[q.id] = std::move(*it);
            it = sv->active.erase(it);
            nfin++;
        } else {
            ++it;
        }
    }
    return nfin;
}

template <class F>
int guarded(edzt_ctx* c, F&& f)
{
    if (!c) return EDZT_ERR_ARG;
    try {
        CK(cudaSetDevice(c->device));
        f();
        c->err.clear();
        return EDZT_OK;
    } catch (const EdztError& e) {
        c->err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        c->err = e.what();
        return EDZT_ERR_CUDA;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// context accessors for the no-allocation entry point (noalloc.cu); none of
// them builds a table or allocates
// ---------------------------------------------------------------------------
int edzt_ctx_device(const edzt_ctx* c) { return c->device; }

cudaStream_t edzt_ctx_stream(const edzt_ctx* c) { return c->stream; }

void edzt_ctx_set_error(edzt_ctx* c, const char* msg) { c->err = msg ? msg : ""; }

void edzt_count_launches(edzt_ctx* c, long long n) { c->launches += n; }

int edzt_ctx_ready_sector(edzt_ctx* c, int nu, int nd, DevSector* S, const char** why)
{
    if (!c->mt.valid) { *why = "no model: call edzt_set_model first"; return EDZT_ERR_STATE; }
    if (!sector_valid(c, nu, nd)) { *why = "electron counts outside [0, nsite]"; return EDZT_ERR_ARG; }
    const int ns = nsite_of(c);
    const bool ready = c->str_tables.count(std::make_pair(ns, nu)) && c->str_tables.count(std::make_pair(ns, nd)) &&
                       c->mt.ops.count(std::make_pair(nu, 0)) && c->mt.ops.count(std::make_pair(nd, 1));
    if (!ready) {
        *why = "the sector's tables are not built on this context: make one allocating call on the sector "
               "first (edzt_hx or edzt_lanczos_iteration)";
        return EDZT_ERR_STATE;
    }
    *S = make_sector(c, nu, nd);   // only looks the tables up
    return EDZT_OK;
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* edzt_version(void) { return "edzt-b200 0.1 (sm_100a)"; }

int edzt_ctx_create(int device, edzt_ctx** out)
{
    if (!out) return EDZT_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return EDZT_ERR_CUDA;
    }
    edzt_ctx* c = new edzt_ctx();
    c->device = device;
    int rc = guarded(c, [&] {
        CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        edzt_init_binomials(device);
        c->sync_words = std::make_unique<DevBuf>(64);
        c->status = std::make_unique<DevBuf>(64);
        c->scal = std::make_unique<DevBuf>(sizeof(double) * 32);
        c->dot_part = std::make_unique<DevBuf>(sizeof(double) * dot_partials_size());
        CK(cudaMallocHost((void**)&c->pinned, sizeof(double) * 32));
        CK(cudaEventCreate(&c->ev0));
        CK(cudaEventCreate(&c->ev1));
        size_t total_b = 0;
        CK(cudaMemGetInfo(&c->free_at_create, &total_b));
    });
    if (rc != EDZT_OK) {
        edzt_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return EDZT_OK;
}

void edzt_ctx_destroy(edzt_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->gs_vec.reset();
    c->pool.release_all();
    if (c->pinned) cudaFreeHost(c->pinned);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* edzt_last_error(const edzt_ctx* c) { return c ? c->err.c_str() : "null context"; }

long long edzt_launch_count(const edzt_ctx* c) { return c ? c->launches.load() : 0; }

int edzt_get_stream(edzt_ctx* c, void** stream)
{
    if (!c || !stream) return EDZT_ERR_ARG;
    *stream = (void*)c->stream;
    return EDZT_OK;
}

int edzt_kernel_stats(edzt_ctx* c, long long* launches, double* ms, double* bytes)
{
    if (!c) return EDZT_ERR_ARG;
    if (launches) *launches = c->st_launches;
    if (ms) *ms = c->st_ms;
    if (bytes) *bytes = c->st_bytes;
    return EDZT_OK;
}

#ifdef EDZT_DEVICE_CHECKS
// Checked builds only: the first failed device bounds check (code, a, b, c).
int edzt_debug_bad(long long* out4)
{
    // first recorded violation of the three kernel modules, in that order
    long long t[4] = {0, 0, 0, 0};
    int (*fns[3])(long long*) = {lz_debug_bad, kernels_debug_bad, tables_debug_bad};
    for (int q = 0; q < 3; q++) {
        fns[q](t);
        if (t[0] != 0) break;
    }
    for (int q = 0; q < 4; q++) out4[q] = t[q];
    return 0;
}
#endif

int edzt_reset_stats(edzt_ctx* c)
{
    if (!c) return EDZT_ERR_ARG;
    c->st_launches = 0;
    c->st_ms = 0.0;
    c->st_bytes = 0.0;
    c->log_ms.clear();
    c->log_bytes.clear();
    c->log_states.clear();
    return EDZT_OK;
}

int edzt_kernel_launch_log(edzt_ctx* c, int max, int* n, double* ms, double* bytes, double* states)
{
    if (!c || !n || max < 0) return EDZT_ERR_ARG;
    const int k = (int)std::min<size_t>((size_t)max, c->log_ms.size());
    for (int i = 0; i < k; i++) {
        if (ms) ms[i] = c->log_ms[i];
        if (bytes) bytes[i] = c->log_bytes[i];
        if (states) states[i] = c->log_states[i];
    }
    *n = k;
    return EDZT_OK;
}

int edzt_set_engine(edzt_ctx* c, int engine)
{
    return guarded(c, [&] {
        arg_check(engine == EDZT_ENGINE_FUSED || engine == EDZT_ENGINE_PLAIN, "unknown engine");
        c->engine = engine;
    });
}

int edzt_set_model(edzt_ctx* c, int norb, int nbath, const double* em, const double* ek, const double* vmk,
                   double U, double Up, double Jex, double Jp, double mu)
{
    return guarded(c, [&] {
        const DevModel m = model_from(norb, nbath, em, ek, vmk, U, Up, Jex, Jp, mu);
        c->has_gs = false;
        set_tables_model(c->mt, m, c->stream);
    });
}

long long edzt_sector_dim(edzt_ctx* c, int ne_up, int ne_dn)
{
    if (!c || !c->mt.valid) return 0;
    return sector_dim(c, ne_up, ne_dn);
}

int edzt_basis(edzt_ctx* c, int ne_up, int ne_dn, int* nup, int* ndn, uint32_t* up, uint32_t* dn)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        StrTable& su = str_table(c, ne_up);
        StrTable& sd = str_table(c, ne_dn);
        if (nup) *nup = su.count;
        if (ndn) *ndn = sd.count;
        if (up) copy_out(c, up, su.str->p, sizeof(uint32_t) * su.count);
        if (dn) copy_out(c, dn, sd.str->p, sizeof(uint32_t) * sd.count);
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_basis_rank(edzt_ctx* c, int ne, int32_t* rank)
{
    return guarded(c, [&] {
        require_model(c);
        arg_check(ne >= 0 && ne <= c->mt.model.nsite && rank != nullptr, "bad electron count or null rank");
        StrTable& s = str_table(c, ne);
        copy_out(c, rank, s.rank->p, sizeof(int32_t) * ((size_t)1 << c->mt.model.nsite));
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_hx(edzt_ctx* c, int ne_up, int ne_dn, const double* x, double* y, int accumulate)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(x != nullptr && y != nullptr, "x and y required");
        DevSector S = make_sector(c, ne_up, ne_dn);
        InVec xi(c, x, S.dim);
        OutVec yo(c, y, S.dim);
        if (accumulate) yo.preload();
        Lease<double> hs(c->pool, (size_t)std::max(hx_scratch_size(S.up.count, S.dn.count), 1LL));
        launch_hx(S, xi.d, yo.d, accumulate ? 1 : 0, hs.p, c->stream);
        c->launches += 2;
        CKLAUNCH();
        yo.finish();
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_apply_c(edzt_ctx* c, int ne_up, int ne_dn, const double* vec, int pm, int iorb, int ispin, double* vec_out)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(pm == 1 || pm == 2, "pm must be 1 or 2");
        arg_check(iorb >= 1 && iorb <= c->mt.model.norb && (ispin == 1 || ispin == 2), "bad iorb/ispin");
        arg_check(vec != nullptr && vec_out != nullptr, "vec and vec_out required");
        int ou, od;
        excitation(ne_up, ne_dn, pm, ispin, &ou, &od);
        arg_check(sector_dim(c, ou, od) > 0, "output sector is empty");
        ApplyCArgs A = applyc_args(c, ne_up, ne_dn, pm, iorb, ispin, ou, od);
        InVec vi(c, vec, sector_dim(c, ne_up, ne_dn));
        OutVec vo(c, vec_out, sector_dim(c, ou, od));
        launch_apply_c(A, vi.d, vo.d, c->stream);
        c->launches += 1;
        CKLAUNCH();
        vo.finish();
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_lanczos_iteration(edzt_ctx* c, int ne_up, int ne_dn, const double* v_init, int maxnstep, int* nstep,
                           double* a, double* b)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(v_init && nstep && a && b && maxnstep >= 1, "bad arguments");
        const long long dim = sector_dim(c, ne_up, ne_dn);
        arg_check(dim > 0, "empty sector");
        InVec vi(c, v_init, dim);
        std::vector<double> ha(maxnstep, 0.0), hb(maxnstep, 0.0);
        if (c->engine == EDZT_ENGINE_FUSED) {
            Lease<double> ab(c->pool, (size_t)2 * maxnstep);
            std::vector<JobSpec> specs(1);
            JobSpec& s = specs[0];
            s.nu = ne_up; s.nd = ne_dn;
            s.mode = LZ_COEFF;
            s.init = LZ_INIT_COPY;
            s.ac_src = vi.d;
            s.maxnstep = maxnstep;
            s.a = ab.p; s.b = ab.p + maxnstep;
            run_jobs(c, specs);
            CK(cudaMemcpyAsync(ha.data(), ab.p, sizeof(double) * maxnstep, cudaMemcpyDeviceToHost, c->stream));
            CK(cudaMemcpyAsync(hb.data(), ab.p + maxnstep, sizeof(double) * maxnstep, cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            *nstep = specs[0].nstep;
        } else {
            DevSector S = make_sector(c, ne_up, ne_dn);
            *nstep = plain_lanczos(c, S, vi.d, maxnstep, ha.data(), hb.data(), nullptr, nullptr, nullptr);
        }
        copy_out(c, a, ha.data(), sizeof(double) * maxnstep);
        copy_out(c, b, hb.data(), sizeof(double) * maxnstep);
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_diag_lanczos(edzt_ctx* c, int ne_up, int ne_dn, int maxnstep, uint64_t seed, uint64_t stream,
                      double* eigval, double* eigvec, double* residual)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(eigval != nullptr && maxnstep >= 1, "bad arguments");
        const long long dim = sector_dim(c, ne_up, ne_dn);
        arg_check(dim > 0, "empty sector");
        // a one-sector ground_state on the requested start-vector stream, always by Lanczos
        std::vector<int> sec = {ne_up, ne_dn};
        int is = 0;
        double e0 = 0.0;
        struct Keep {
            edzt_ctx* c;
            int solver;
            ~Keep() { c->diag_solver = solver; }
        } keep{c, c->diag_solver};
        c->diag_solver = EDZT_DIAG_LANCZOS;
        ground_state_impl(c, 1, sec.data(), maxnstep, seed, &is, &e0, nullptr, nullptr, &stream);
        *eigval = e0;
        if (eigvec) copy_out(c, eigvec, c->gs_vec.p, sizeof(double) * dim);
        if (residual) *residual = c->gs_residual;
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_diag_arpack(edzt_ctx* c, int ne_up, int ne_dn, uint64_t seed, uint64_t stream, double* eigval,
                     double* eigvec, double* ritz, double* resid, int* nmult)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(eigval != nullptr, "eigval required");
        const long long dim = sector_dim(c, ne_up, ne_dn);
        arg_check(dim > 0, "empty sector");
        DevSector S = make_sector(c, ne_up, ne_dn);
        Lease<double> vec(c->pool, (size_t)dim);
        ArpackOut R;
        diag_arpack_impl(c, S, edzt_stream_key(seed, stream), vec.p, R, resid != nullptr);
        *eigval = R.eigval;
        for (int i = 0; i < kArNev; i++) {
            if (ritz) ritz[i] = R.ritz[i];
            if (resid) resid[i] = R.resid[i];
        }
        if (nmult) *nmult = R.nmult;
        if (eigvec) copy_out(c, eigvec, vec.p, sizeof(double) * dim);
        CK(cudaStreamSynchronize(c->stream));
    });
}

int edzt_set_diag_solver(edzt_ctx* c, int diag_solver)
{
    return guarded(c, [&] {
        if (diag_solver != EDZT_DIAG_LANCZOS && diag_solver != EDZT_DIAG_ARPACK)
            throw EdztError{EDZT_ERR_ARG, "invalid diag solver"};
        c->diag_solver = diag_solver;
    });
}

int edzt_set_keep_vectors(edzt_ctx* c, int keep)
{
    return guarded(c, [&] {
        if (keep != 0 && keep != 1) throw EdztError{EDZT_ERR_ARG, "keep must be 0 or 1"};
        c->keep_vectors = keep;
    });
}

int edzt_ground_state(edzt_ctx* c, int nsector, const int* sectors, int maxnstep, uint64_t seed, int* isector,
                      double* e0, double* gsvec, double* e_sector)
{
    return guarded(c, [&] {
        arg_check(isector != nullptr && e0 != nullptr, "isector and e0 required");
        ground_state_impl(c, nsector, sectors, maxnstep, seed, isector, e0, gsvec, e_sector);
    });
}

long long edzt_gs_dim(edzt_ctx* c)
{
    if (!c || !c->has_gs) return 0;
    return sector_dim(c, c->gs_up, c->gs_dn);
}

int edzt_green_diag(edzt_ctx* c, int iorb, int ispin, int maxnstep, int nw, const double* omega, double* ap,
                    double* bp, double* am, double* bm, double* g)
{
    return guarded(c, [&] {
        arg_check(ap && bp && am && bm && g && (omega || nw == 0), "bad arguments");
        green_diag_impl(c, iorb, ispin, maxnstep, nw, omega, ap, bp, am, bm, g);
    });
}

int edzt_green_real(edzt_ctx* c, int iorb, int ispin, int maxnstep, int nw, const double* omega, double eta,
                    double* g)
{
    return guarded(c, [&] {
        arg_check(g != nullptr && (omega || nw == 0) && eta > 0.0, "bad arguments (eta > 0)");
        green_diag_impl(c, iorb, ispin, maxnstep, nw, omega, nullptr, nullptr, nullptr, nullptr, g, 1, eta);
    });
}

int edzt_gs_occupancy(edzt_ctx* c, int nspin, double* occ, double* docc)
{
    return guarded(c, [&] {
        require_model(c);
        require_gs(c);
        arg_check(nspin == 1 || nspin == 2, "nspin must be 1 or 2");
        const int norb = c->mt.model.norb;
        StrTable& su = str_table(c, c->gs_up);
        StrTable& sd = str_table(c, c->gs_dn);
        const long long dim = (long long)su.count * sd.count;
        Lease<double> part(c->pool, (size_t)occ_partials_size());
        launch_gs_occ(c->gs_vec.p, su.str->as<uint32_t>(), sd.str->as<uint32_t>(), su.count, dim, norb, part.p,
                      c->stream);
        c->launches += 1;
        CKLAUNCH();
        std::vector<double> hp((size_t)occ_partials_size());
        CK(cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        double sum[12] = {0.0};
        for (size_t b = 0; b < hp.size() / 12; b++)
            for (int q = 0; q < 12; q++) sum[q] += hp[b * 12 + q];
        for (int ispin = 0; ispin < nspin; ispin++)
            for (int a = 0; a < norb; a++)
                if (occ) occ[a + norb * ispin] = sum[4 * ispin + a];
        if (docc)
            for (int a = 0; a < norb; a++) docc[a] = sum[8 + a];
    });
}

int edzt_cluster_green_matrix(edzt_ctx* c, int nspin, int maxnstep, int nw, const double* omega, double* G)
{
    return guarded(c, [&] {
        arg_check(G != nullptr && (omega || nw == 0), "bad arguments");
        cluster_green_matrix_impl(c, nspin, maxnstep, nw, omega, G);
    });
}

int edzt_cluster_green_ftn(edzt_ctx* c, int nspin, int maxnstep, int nw, const double* omega, double* G_cl,
                           double* coeffs)
{
    return guarded(c, [&] {
        arg_check(G_cl != nullptr && (omega || nw == 0), "bad arguments");
        cluster_green_impl(c, nspin, maxnstep, nw, omega, G_cl, coeffs);
    });
}

int edzt_server_create(edzt_ctx* c, int maxnstep, int nw, const double* omega, size_t hbm_budget,
                       edzt_server** out)
{
    if (!out) return EDZT_ERR_ARG;
    *out = nullptr;
    return guarded(c, [&] {
        arg_check(maxnstep >= 1 && nw >= 0 && (nw == 0 || omega != nullptr), "maxnstep >= 1, nw >= 0, omega");
        auto sv = std::make_unique<edzt_server>();
        sv->c = c;
        sv->maxnstep = maxnstep;
        sv->nw = nw;
        sv->omega = std::make_unique<DevBuf>(sizeof(double) * std::max(nw, 1));
        if (nw > 0) CK(cudaMemcpy(sv->omega->p, omega, sizeof(double) * nw, cudaMemcpyDefault));
        if (hbm_budget == 0) {
            size_t fr = 0, tot = 0;
            CK(cudaMemGetInfo(&fr, &tot));
            hbm_budget = fr / 10 * 8;
        }
        sv->budget = (long long)hbm_budget;
        *out = sv.release();
    });
}

int edzt_server_submit(edzt_server* sv, const edzt_instance* inst, long long* id)
{
    if (!sv) return EDZT_ERR_ARG;
    return guarded(sv->c, [&] {
        arg_check(inst != nullptr && id != nullptr, "inst and id required");
        auto q = std::make_unique<ServReq>();
        init_inst(*inst, q->I);
        if (q->I.footprint > sv->budget)
            throw EdztError{EDZT_ERR_OOM, "request needs " + std::to_string(q->I.footprint) +
                                              " bytes of device memory, the server's budget is " +
                                              std::to_string(sv->budget)};
        q->id = sv->next_id++;
        *id = q->id;
        sv->queue.push_back(std::move(q));
    });
}

int edzt_server_step(edzt_server* sv, int* nactive, int* nqueued, int* nfinished)
{
    if (!sv) return EDZT_ERR_ARG;
    return guarded(sv->c, [&] {
        const int nf = server_step(sv);
        if (nfinished) *nfinished = nf;
        if (nactive) *nactive = (int)sv->active.size();
        if (nqueued) *nqueued = (int)sv->queue.size();
    });
}

int edzt_tune_sector(edzt_ctx* c, int ne_up, int ne_dn, int steps, int* wc, int* rows, int* block,
                     double* ms_per_step)
{
    return guarded(c, [&] {
        require_model(c);
        check_sector(c, ne_up, ne_dn);
        arg_check(steps >= 2 && steps <= 1000, "steps in [2, 1000]");
        arg_check(sector_dim(c, ne_up, ne_dn) > 0, "empty sector");
        const edzt_ctx::Tuned t = tune_sector(c, ne_up, ne_dn, steps);
        if (wc) *wc = t.wc;
        if (rows) *rows = t.r;
        if (block) *block = t.block;
        if (ms_per_step) *ms_per_step = t.ms_per_step;
    });
}

int edzt_clear_tuning(edzt_ctx* c)
{
    return guarded(c, [&] { c->tuned.clear(); });
}

int edzt_server_set_step_ms(edzt_server* sv, double ms)
{
    if (!sv) return EDZT_ERR_ARG;
    return guarded(sv->c, [&] {
        arg_check(ms > 0.0 && std::isfinite(ms), "step time budget must be a positive number of ms");
        sv->step_ms = ms;
    });
}

int edzt_server_result(edzt_server* sv, long long id, int* done, int* isector, double* e0, double* G_cl)
{
    if (!sv) return EDZT_ERR_ARG;
    return guarded(sv->c, [&] {
        arg_check(done != nullptr, "done required");
        auto it = sv->finished.find(id);
        *done = 0;
        if (it == sv->finished.end()) return;
        ServReq& q = *it->second;
        if (!q.error.empty()) {
            const std::string msg = "request " + std::to_string(id) + ": " + q.error;
            sv->finished.erase(it);
            throw EdztError{EDZT_ERR_NUMERIC, msg};
        }
        *done = 1;
        if (isector) *isector = q.I.best;
        if (e0) *e0 = q.I.e0;
        if (G_cl && !q.G.empty()) copy_out(sv->c, G_cl, q.G.data(), sizeof(double) * q.G.size());
        CK(cudaStreamSynchronize(sv->c->stream));
        sv->finished.erase(it);
    });
}

int edzt_server_cancel(edzt_server* sv, long long id)
{
    if (!sv) return EDZT_ERR_ARG;
    return guarded(sv->c, [&] {
        for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it)
            if ((*it)->id == id) {
                sv->queue.erase(it);
                return;
            }
        for (auto& q : sv->active)
            if (q->id == id) {
                q->cancelled = true;   // retired, its memory released, at the next step
                return;
            }
        throw EdztError{EDZT_ERR_ARG, "no queued or running request " + std::to_string(id)};
    });
}

int edzt_instance_footprint(const edzt_instance* inst, long long* bytes)
{
    if (!inst || !bytes) return EDZT_ERR_ARG;
    try {
        BatchInst I;
        init_inst(*inst, I);
        *bytes = I.footprint;
        return EDZT_OK;
    } catch (const EdztError& e) {
        return e.code;
    }
}

int edzt_set_fault_test(edzt_ctx* c, int pass_cap, double wait_seconds, int stall_cta)
{
    return guarded(c, [&] {
        arg_check(pass_cap >= 0 && wait_seconds >= 0.0 && stall_cta >= -1, "bad fault-test settings");
        c->dbg_pass_cap = pass_cap;
        c->dbg_wait_ns = (unsigned long long)(wait_seconds * 1e9);
        c->dbg_stall_cta = stall_cta;
    });
}

void edzt_server_destroy(edzt_server* sv)
{
    if (!sv) return;
    cudaSetDevice(sv->c->device);
    cudaStreamSynchronize(sv->c->stream);
    delete sv;
}

int edzt_solve_batch(edzt_ctx* c, int ninst, const edzt_instance* inst, int maxnstep, int nw, const double* omega,
                     int* isector, double* e0, double* G_cl, size_t hbm_budget)
{
    return guarded(c, [&] { solve_batch_impl(c, ninst, inst, maxnstep, nw, omega, isector, e0, G_cl, hbm_budget); });
}

int edzt_solve(edzt_ctx* c, int nsector, const int* sectors, int maxnstep, uint64_t seed, int nspin, int nw,
               const double* omega, int* isector, double* e0, double* G_cl, double* coeffs)
{
    return guarded(c, [&] {
        arg_check(isector && e0 && G_cl && (omega || nw == 0), "bad arguments");
        ground_state_impl(c, nsector, sectors, maxnstep, seed, isector, e0, nullptr, nullptr);
        cluster_green_impl(c, nspin, maxnstep, nw, omega, G_cl, coeffs);
    });
}

}  // extern "C"
