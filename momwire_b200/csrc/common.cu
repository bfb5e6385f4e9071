// Host-side helpers shared by every translation unit: error text, version,
// Gauss-Legendre tables.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace mw {

static thread_local char g_err[512] = "";
static std::atomic<int64_t> g_launches{0};

void count_launch(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

mw_status cuda_status(cudaError_t e, const char* what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return MW_ERR_CUDA;
}

// Gauss-Legendre on [0,1]: Newton iteration on the Legendre recurrence,
// started from the Chebyshev-like guess cos(pi (i + 3/4) / (n + 1/2)).
static void compute_gl(int n, std::vector<double>& t, std::vector<double>& w) {
    t.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            double pn = (n == 1) ? x : p1;
            double pm = (n == 1) ? 1.0 : p0;
            dp = n * (x * pn - pm) / (x * x - 1.0);
            double dx = pn / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-17) break;
        }
        // recompute derivative at the converged node
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k) {
            double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        double pn = (n == 1) ? x : p1, pm = (n == 1) ? 1.0 : p0;
        dp = n * (x * pn - pm) / (x * x - 1.0);
        double wi = 2.0 / ((1.0 - x * x) * dp * dp);
        // ascending order on [0,1]
        t[n - 1 - i] = 0.5 * (x + 1.0);
        w[n - 1 - i] = 0.5 * wi;
    }
}

void gauss_legendre01(int n, const double** t, const double** w) {
    static std::mutex mu;
    static std::vector<double> T[33], W[33];
    std::lock_guard<std::mutex> g(mu);
    if (n < 1) n = 1;
    if (n > 32) n = 32;
    if (T[n].empty()) compute_gl(n, T[n], W[n]);
    *t = T[n].data();
    *w = W[n].data();
}

// ------------------------------------------------------------- profiling
struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    double flops, bytes;
};

static std::mutex g_prof_mu;
static bool g_prof_on = false;
static std::vector<ProfRec> g_prof_pending;
static std::vector<cudaEvent_t> g_prof_pool;
static int64_t g_prof_count[PC_COUNT];
static double g_prof_ms[PC_COUNT], g_prof_flops[PC_COUNT], g_prof_bytes[PC_COUNT];

static cudaEvent_t prof_event() {
    if (!g_prof_pool.empty()) {
        cudaEvent_t e = g_prof_pool.back();
        g_prof_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

ProfileScope::ProfileScope(int cls, cudaStream_t st, double flops, double bytes)
    : cls_(cls), st_(st), flops_(flops), bytes_(bytes), rec_(nullptr) {
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (!g_prof_on) return;
    ProfRec* r = new ProfRec{cls, prof_event(), prof_event(), flops, bytes};
    cudaEventRecord(r->a, st);
    rec_ = r;
}

ProfileScope::~ProfileScope() {
    if (!rec_) return;
    ProfRec* r = static_cast<ProfRec*>(rec_);
    cudaEventRecord(r->b, st_);
    std::lock_guard<std::mutex> g(g_prof_mu);
    g_prof_pending.push_back(*r);
    delete r;
}

static void prof_drain() {
    for (auto& r : g_prof_pending) {
        cudaEventSynchronize(r.b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        g_prof_count[r.cls] += 1;
        g_prof_ms[r.cls] += ms;
        g_prof_flops[r.cls] += r.flops;
        g_prof_bytes[r.cls] += r.bytes;
        g_prof_pool.push_back(r.a);
        g_prof_pool.push_back(r.b);
    }
    g_prof_pending.clear();
}

}  // namespace mw

extern "C" void mw_profile_enable(int32_t on) {
    std::lock_guard<std::mutex> g(mw::g_prof_mu);
    mw::prof_drain();
    mw::g_prof_on = on != 0;
    for (int i = 0; i < mw::PC_COUNT; ++i) {
        mw::g_prof_count[i] = 0;
        mw::g_prof_ms[i] = mw::g_prof_flops[i] = mw::g_prof_bytes[i] = 0.0;
    }
}

extern "C" int32_t mw_profile_read(int32_t cls, int64_t* launches, double* total_ms, double* flops, double* bytes) {
    std::lock_guard<std::mutex> g(mw::g_prof_mu);
    if (cls < 0 || cls >= mw::PC_COUNT) return MW_ERR_INVALID;
    mw::prof_drain();
    if (launches) *launches = mw::g_prof_count[cls];
    if (total_ms) *total_ms = mw::g_prof_ms[cls];
    if (flops) *flops = mw::g_prof_flops[cls];
    if (bytes) *bytes = mw::g_prof_bytes[cls];
    return MW_OK;
}

extern "C" int32_t mw_version(void) { return 100; }  // 0.1.0

extern "C" const char* mw_last_error(void) { return mw::g_err; }

extern "C" int64_t mw_launch_count(void) { return mw::g_launches.load(std::memory_order_relaxed); }
