// C++ drop-in facade: the reference's hostLibrary entry points over the C-ABI.
//
// Output layout, precision and error behaviour follow Library/hostLibrary.cu
// (lines cited per function).  Numbers are formatted as "%.*g" / "%d" -- what
// std::ostream's default float field uses, so the bytes are identical to the
// reference's `outFileStream << value` at the same precision -- by
// std::to_chars (general format with a precision is specified as printf's %.*g;
// tests compare the bytes with printf-style formatting).  2-D maps are formatted
// by several threads in blocks and written in order: the text of value i is
// determined by i alone (", " before every value but the first, "\n" before
// each new row), so the file is the same bytes as the serial rule produces.
#include <cuda_runtime.h>
#include <math.h>
#include <sched.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <charconv>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/cbf.h"
#include "../../include/hostLibrary.h"

namespace {

std::atomic<int> g_system{-1};
std::mutex g_path_mu;
std::string g_path;
bool g_path_set = false;

int system_from_env()
{
    const char* s = getenv("CBF_SYSTEM");
    if (!s || !*s) return CBF_SYS_MEMRISTIVE5;
    if (!strcmp(s, "memristive5")) return CBF_SYS_MEMRISTIVE5;
    if (!strcmp(s, "rossler")) return CBF_SYS_ROSSLER;
    if (!strcmp(s, "lorenz")) return CBF_SYS_LORENZ;
    if (!strcmp(s, "chen")) return CBF_SYS_CHEN;
    char* end = nullptr;
    long v = strtol(s, &end, 10);
    if (end && *end == 0 && v >= 0 && v < CBF_NUM_SYSTEMS) return (int)v;
    fprintf(stderr, "CBF_SYSTEM=%s is not a known system; using memristive5\n", s);
    return CBF_SYS_MEMRISTIVE5;
}

int current_system()
{
    int s = g_system.load();
    if (s < 0) {
        s = system_from_env();
        g_system.store(s);
    }
    return s;
}

// Surrogate-refined LLE2D: -1 = the environment's CBF_SURROGATE decides.
std::atomic<int> g_surrogate{-1};

bool surrogate_enabled()
{
    const int v = g_surrogate.load();
    if (v >= 0) return v != 0;
    const char* e = getenv("CBF_SURROGATE");
    return e && *e && strcmp(e, "0") != 0;
}

std::string current_path()
{
    std::lock_guard<std::mutex> lk(g_path_mu);
    if (g_path_set) return g_path;
    const char* e = getenv("CBF_OUT_FILE_PATH");
    return (e && *e) ? std::string(e) : std::string("mat.csv");
}

// gpuAssert (cudaMacros.cu:3-10): print and exit with the code.
[[noreturn]] void fatal(cbf_status st, const char* file, int line)
{
    fprintf(stderr, "GPUassert: %s %s %d\n", cbf_last_error(), file, line);
    exit((int)st);
}

#define CBF_CHECK(call)                                   \
    do {                                                  \
        cbf_status st_ = (call);                          \
        if (st_ != CBF_OK) fatal(st_, __FILE__, __LINE__); \
    } while (0)

// An output file that cannot be written: hostLibrary.cu:134-138.
void io_check(cbf_status st)
{
    if (st == CBF_ERR_IO) {
        printf("\nOutput file open error\n");
        exit(1);
    }
    if (st != CBF_OK) fatal(st, __FILE__, __LINE__);
}

// getValueByIdx (cudaLibrary.cu:210-216) evaluated on the host, as the
// reference does for the 1-D CSV rows (hostLibrary.cu:131-132).
double host_value_by_idx(int idx, int nPts, double start, double finish, int valueNumber)
{
    float p = powf((float)nPts, (float)valueNumber);
    float q = (float)idx / p;
    int cell = ((int)q) % nPts;
    return start + (double)cell * ((double)(finish - start) / (double)(nPts - 1));
}

// Buffered CSV writer.  `open` failure is reported at the first value, like the
// reference's per-value `is_open()` check (hostLibrary.cu:534-551).
class CsvOut {
public:
    explicit CsvOut(const std::string& path, bool append = false)
    {
        f_ = fopen(path.c_str(), append ? "ab" : "wb");
        buf_.reserve(1 << 20);
    }
    ~CsvOut() { close(); }
    bool is_open() const { return f_ != nullptr; }
    void precision(int p) { prec_ = p; }
    void str(const char* s)
    {
        if (!f_) return;
        buf_.append(s);
        maybe_flush();
    }
    void dbl(double v)
    {
        if (!f_) return;
        char tmp[64];
        const auto r = std::to_chars(tmp, tmp + sizeof(tmp), v, std::chars_format::general, prec_);
        buf_.append(tmp, (size_t)(r.ptr - tmp));
        maybe_flush();
    }
    void i32(int v)
    {
        if (!f_) return;
        char tmp[16];
        const auto r = std::to_chars(tmp, tmp + sizeof(tmp), v);
        buf_.append(tmp, (size_t)(r.ptr - tmp));
        maybe_flush();
    }
    int precision() const { return prec_; }
    // The underlying file with everything buffered so far written out.
    FILE* file()
    {
        if (f_) flush();
        return f_;
    }
    void close()
    {
        if (f_) {
            flush();
            fclose(f_);
            f_ = nullptr;
        }
    }

private:
    void maybe_flush()
    {
        if (buf_.size() >= (1u << 20)) flush();
    }
    void flush()
    {
        if (!buf_.empty()) fwrite(buf_.data(), 1, buf_.size(), f_);
        buf_.clear();
    }
    FILE* f_ = nullptr;
    std::string buf_;
    int prec_ = 6;
};

// Map header "r0 r1\nr2 r3\n" (hostLibrary.cu:476-480).
void write_header(CsvOut& out, const double* ranges)
{
    if (!out.is_open()) return;
    out.dbl(ranges[0]);
    out.str(" ");
    out.dbl(ranges[1]);
    out.str("\n");
    out.dbl(ranges[2]);
    out.str(" ");
    out.dbl(ranges[3]);
    out.str("\n");
}

// Map values in index order with the reference's row-break rule
// (hostLibrary.cu:534-546): ", " before every value but the first, "\n" before
// the first of each new row -- so the text of value i depends on i alone.
// Values [i0, i1) of a map with their separators, appended to `out`.
template <class T>
void format_map_range(const T* v, long long i0, long long i1, int nPts, int prec, std::string& out)
{
    char tmp[64];
    for (long long i = i0; i < i1; ++i) {
        if (i > 0) {
            out.append(", ", 2);
            if (i % nPts == 0) out.push_back('\n');
        }
        std::to_chars_result r;
        if constexpr (std::is_same<T, double>::value)
            r = std::to_chars(tmp, tmp + sizeof(tmp), v[i], std::chars_format::general, prec);
        else
            r = std::to_chars(tmp, tmp + sizeof(tmp), v[i]);
        out.append(tmp, (size_t)(r.ptr - tmp));
    }
}

// Threads for the map formatter: CBF_CSV_THREADS if > 0, else the CPUs this
// process may run on (<= 64).
int csv_threads()
{
    const char* e = getenv("CBF_CSV_THREADS");
    int t = (e && *e) ? atoi(e) : 0;
    if (t <= 0) {
        cpu_set_t set;
        CPU_ZERO(&set);
        t = sched_getaffinity(0, sizeof(set), &set) == 0 ? CPU_COUNT(&set)
                                                          : (int)std::thread::hardware_concurrency();
    }
    return std::max(1, std::min(t, 64));
}

// The whole map after the header: rounds of `threads` blocks of kBlock values,
// each block formatted by its own thread; the previous round's text is written
// (in index order) by one more thread while the next round is formatted.
template <class T>
void write_map_parallel(CsvOut& out, const T* v, long long n, int nPts)
{
    FILE* f = out.file();
    if (!f || n <= 0) return;
    constexpr long long kBlock = 1 << 18;
    const int threads = csv_threads();
    const int prec = out.precision();
    if (threads == 1 || n <= kBlock) {
        std::string buf;
        for (long long i0 = 0; i0 < n; i0 += kBlock) {
            buf.clear();
            format_map_range(v, i0, std::min(n, i0 + kBlock), nPts, prec, buf);
            fwrite(buf.data(), 1, buf.size(), f);
        }
        return;
    }
    std::vector<std::string> bufs[2] = {std::vector<std::string>((size_t)threads),
                                        std::vector<std::string>((size_t)threads)};
    std::thread writer;
    int side = 0;
    for (long long base = 0; base < n; base += kBlock * threads, side ^= 1) {
        const int used = (int)std::min<long long>(threads, (n - base + kBlock - 1) / kBlock);
        std::vector<std::string>& cur = bufs[side];
        auto work = [&, base](int t) {
            const long long i0 = base + (long long)t * kBlock;
            cur[(size_t)t].clear();
            format_map_range(v, i0, std::min(n, i0 + kBlock), nPts, prec, cur[(size_t)t]);
        };
        std::vector<std::thread> pool;
        pool.reserve((size_t)used);
        for (int t = 0; t < used; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
        if (writer.joinable()) writer.join();  // the previous round is on disk
        writer = std::thread([f, &cur, used] {
            for (int t = 0; t < used; ++t) fwrite(cur[(size_t)t].data(), 1, cur[(size_t)t].size(), f);
        });
    }
    if (writer.joinable()) writer.join();
}

void bif1d_common(bool ic, double tMax, int nPts, double h, int nIC, const double* icv,
                  const double* ranges, const int* idx, int wv, double maxValue,
                  double transientTime, const double* values, int nV, int preScaller)
{
    cbf_job job;
    cbf_job_init(&job);
    job.task = CBF_TASK_PEAKS;
    job.system = current_system();
    job.sweepIC = ic ? 1 : 0;
    job.dims = 1;
    job.nPts = nPts;
    job.h = h;
    job.tMax = tMax;
    job.transientTime = transientTime;
    job.maxValue = maxValue;
    job.writableVar = wv;
    job.preScaller = preScaller;
    job.nIC = nIC;
    job.nV = nV;
    job.ranges[0] = ranges[0];
    job.ranges[1] = ranges[1];
    job.idxMut[0] = idx[0];
    for (int i = 0; i < nIC && i < CBF_MAX_DIM; ++i) job.ic[i] = icv[i];
    for (int i = 0; i < nV && i < CBF_MAX_VALUES; ++i) job.values[i] = values[i];
    CBF_CHECK(cbf_validate(&job));
    const int cap = cbf_peak_capacity(&job);
    job.peakCapacity = cap;

    // Bounded host/device footprint: process the points in chunks.
    const size_t budget = (size_t)1 << 30;
    long long chunk = (long long)(budget / ((size_t)cap * sizeof(double)));
    if (chunk < 1) chunk = 1;
    if (chunk > nPts) chunk = nPts;
    std::vector<double> peaks((size_t)chunk * cap);
    std::vector<int32_t> counts((size_t)chunk);

    const std::string path = current_path();
    int append = 0;
    for (long long first = 0; first < nPts; first += chunk) {
        const long long n = (first + chunk <= nPts) ? chunk : nPts - first;
        job.firstPoint = first;
        job.nPoints = n;
        CBF_CHECK(cbf_run_host(&job, peaks.data(), counts.data()));
        io_check(cbf_csv_write_peaks(path.c_str(), nPts, ranges, first, n, peaks.data(), cap,
                                     counts.data(), append));
        append = 1;
    }
}

void map2d_common(bool ic, int task, double tMax, int nPts, double h, int nIC, const double* icv,
                  const double* ranges, const int* idx, int wv, double maxValue, int maxPeaks,
                  double transientTime, const double* values, int nV, int preScaller,
                  int kdeSampling, double i1, double i2, double smooth, double eps,
                  bool header, int precision)
{
    std::vector<int32_t> res((size_t)nPts * (size_t)nPts);
    cbf_status st;
    if (task == CBF_TASK_KDE) {
        st = (ic ? cbf_bifurcation2d_kde_ic : cbf_bifurcation2d_kde)(
            current_system(), tMax, nPts, h, nIC, icv, ranges, idx, wv, maxValue, maxPeaks,
            transientTime, values, nV, preScaller, kdeSampling, i1, i2, smooth, res.data());
    } else {
        st = (ic ? cbf_bifurcation2d_dbscan_ic : cbf_bifurcation2d_dbscan)(
            current_system(), tMax, nPts, h, nIC, icv, ranges, idx, wv, maxValue, maxPeaks,
            transientTime, values, nV, preScaller, eps, res.data());
    }
    CBF_CHECK(st);
    io_check(cbf_csv_write_map(current_path().c_str(), res.data(), 0, (int64_t)res.size(), nPts,
                               header ? ranges : nullptr, precision));
}

// Chunk size the reference used for the LLE launch; its seed index is local to
// the chunk (cudaLibrary.cu:695,723).  LLE1D/LLE1DIC: free/4 / (8*blocks)
// (hostLibrary.cu:1295-1298); LLE2D: 200000 (:1552); LLE2DIC: 0.95*free/(8*blocks)
// (:1691-1696).
long long reference_seed_chunk(int variant, double tMax, double NT, int nPts)
{
    const long long total = variant >= 2 ? (long long)nPts * nPts : nPts;
    if (variant == 2) return total < 200000 ? total : 200000;
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return 0;
    const int blocks = (int)(tMax / NT);
    if (blocks <= 0) return 0;
    size_t f = freeB;
    if (variant == 3)
        f = (size_t)((double)f * 0.95);
    else
        f /= 4;
    long long lim = (long long)(f / (sizeof(double) * (size_t)blocks));
    if (lim > total) lim = total;
    return lim > 0 ? lim : 1;
}

void lle_common(int variant, double tMax, double NT, int nPts, double h, double eps,
                const double* icv, int nIC, const double* ranges, const int* idx, int wv,
                double maxValue, double transientTime, const double* values, int nV)
{
    const bool ic = (variant == 1 || variant == 3);
    const int dims = variant >= 2 ? 2 : 1;
    const long long total = dims == 2 ? (long long)nPts * nPts : nPts;
    std::vector<double> res((size_t)(total > 0 ? total : 0));
    const long long seedChunk = reference_seed_chunk(variant, tMax, NT, nPts);
    if (variant == 2 && surrogate_enabled()) {
        // the opt-in surrogate-refined map (same grid, seeds and layout) plus its classes
        std::vector<int32_t> cls((size_t)(total > 0 ? total : 0));
        CBF_CHECK(cbf_lle2d_surrogate(current_system(), tMax, NT, nPts, h, eps, icv, nIC, ranges, idx, wv,
                                      maxValue, transientTime, values, nV, seedChunk, nullptr, nullptr,
                                      res.data(), cls.data(), nullptr));
        const std::string path = current_path();
        io_check(cbf_csv_write_map(path.c_str(), res.data(), 1, total, nPts, ranges, 6));
        io_check(cbf_csv_write_map((path + ".regime.csv").c_str(), cls.data(), 0, total, nPts, ranges, 6));
        return;
    }
    cbf_status st;
    if (dims == 1)
        st = (ic ? cbf_lle1d_ic : cbf_lle1d)(current_system(), tMax, NT, nPts, h, eps, icv, nIC, ranges,
                                            idx, wv, maxValue, transientTime, values, nV, seedChunk,
                                            res.data());
    else
        st = (ic ? cbf_lle2d_ic : cbf_lle2d)(current_system(), tMax, NT, nPts, h, eps, icv, nIC, ranges,
                                            idx, wv, maxValue, transientTime, values, nV, seedChunk,
                                            res.data());
    CBF_CHECK(st);
    const std::string path = current_path();
    if (dims == 1)
        io_check(cbf_csv_write_pairs(path.c_str(), nPts, ranges, res.data(), total, 6));
    else  // LLE2DIC has no header (hostLibrary.cu:1732-1788)
        io_check(cbf_csv_write_map(path.c_str(), res.data(), 1, total, nPts,
                                   variant == 2 ? ranges : nullptr, 6));
}

// Chunk of the reference's LS launches, to which its seed index is local:
// min(points, (free/4) / (8 * blocks * nIC)) (hostLibrary.cu:1820-1826, :1945-1951).
long long ls_seed_chunk(int dims, double tMax, double NT, int nPts, int nIC)
{
    const long long total = dims == 2 ? (long long)nPts * nPts : nPts;
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return 0;
    const int blocks = (int)(tMax / NT);
    if (blocks <= 0 || nIC <= 0) return 0;
    long long lim = (long long)((freeB / 4) / (sizeof(double) * (size_t)blocks * (size_t)nIC));
    if (lim > total) lim = total;
    return lim > 0 ? lim : 1;
}

void ls_common(int dims, double tMax, double NT, int nPts, double h, double eps, const double* icv,
               int nIC, const double* ranges, const int* idx, int wv, double maxValue,
               double transientTime, const double* values, int nV)
{
    const long long total = dims == 2 ? (long long)nPts * nPts : nPts;
    const int cols = nIC > 0 ? nIC : 0;
    std::vector<double> res((size_t)(total > 0 ? total : 0) * (size_t)cols);
    const long long seedChunk = ls_seed_chunk(dims, tMax, NT, nPts, nIC);
    const cbf_status st = (dims == 1 ? cbf_ls1d : cbf_ls2d)(current_system(), tMax, NT, nPts, h, eps, icv,
                                                           nIC, ranges, idx, wv, maxValue, transientTime,
                                                           values, nV, seedChunk, res.data());
    CBF_CHECK(st);
    const std::string path = current_path();
    if (dims == 1) {
        io_check(cbf_csv_write_rows(path.c_str(), nPts, ranges, res.data(), total, cols, 6));
        return;
    }
    std::vector<double> col((size_t)(total > 0 ? total : 0));
    for (int k = 0; k < cols; ++k) {
        for (long long m = 0; m < total; ++m) col[(size_t)m] = res[(size_t)m * cols + k];
        const std::string p = path + std::to_string(k + 1) + ".csv";
        io_check(cbf_csv_write_map(p.c_str(), col.data(), 1, total, nPts, ranges, 6));
    }
}

}  // namespace

// hostLibrary.cu:7-158
void bifurcation1D(const double tMax, const int nPts, const double h,
                   const int amountOfInitialConditions, const double* initialConditions,
                   const double* ranges, const int* indicesOfMutVars, const int writableVar,
                   const double maxValue, const double transientTime, const double* values,
                   const int amountOfValues, const int preScaller)
{
    bif1d_common(false, tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                 indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues,
                 preScaller);
}

// hostLibrary.cu:243-393
void bifurcation1DIC(const double tMax, const int nPts, const double h,
                     const int amountOfInitialConditions, const double* initialConditions,
                     const double* ranges, const int* indicesOfMutVars, const int writableVar,
                     const double maxValue, const double transientTime, const double* values,
                     const int amountOfValues, const int preScaller)
{
    bif1d_common(true, tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                 indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues,
                 preScaller);
}

// hostLibrary.cu:397-567: header at precision 12 (:474-480)
void bifurcation2DKDE(const double tMax, const int nPts, const double h,
                      const int amountOfInitialConditions, const double* initialConditions,
                      const double* ranges, const int* indicesOfMutVars, const int writableVar,
                      const double maxValue, const int maxAmountOfPeaks,
                      const double transientTime, const double* values,
                      const int amountOfValues, const int preScaller, const int in_kdeSampling,
                      const double in_kdeSamplesInterval1, const double in_kdeSamplesInterval2,
                      const double in_kdeSamplesSmooth)
{
    map2d_common(false, CBF_TASK_KDE, tMax, nPts, h, amountOfInitialConditions, initialConditions,
                 ranges, indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks, transientTime,
                 values, amountOfValues, preScaller, in_kdeSampling, in_kdeSamplesInterval1,
                 in_kdeSamplesInterval2, in_kdeSamplesSmooth, 0.0, true, 12);
}

// hostLibrary.cu:571-744: header at default precision (:651-655)
void bifurcation2DDBSCAN(const double tMax, const int nPts, const double h,
                         const int amountOfInitialConditions, const double* initialConditions,
                         const double* ranges, const int* indicesOfMutVars, const int writableVar,
                         const double maxValue, const int maxAmountOfPeaks,
                         const double transientTime, const double* values,
                         const int amountOfValues, const int preScaller, const double eps)
{
    map2d_common(false, CBF_TASK_DBSCAN, tMax, nPts, h, amountOfInitialConditions,
                 initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                 maxAmountOfPeaks, transientTime, values, amountOfValues, preScaller, 0, 0.0, 0.0,
                 0.0, eps, true, 6);
}

// hostLibrary.cu:929-1090: no header (:1004-1079)
void bifurcation2DKDEIC(const double tMax, const int nPts, const double h,
                        const int amountOfInitialConditions, const double* initialConditions,
                        const double* ranges, const int* indicesOfMutVars, const int writableVar,
                        const double maxValue, const int maxAmountOfPeaks,
                        const double transientTime, const double* values,
                        const int amountOfValues, const int preScaller, const int in_kdeSampling,
                        const double in_kdeSamplesInterval1, const double in_kdeSamplesInterval2,
                        const double in_kdeSamplesSmooth)
{
    map2d_common(true, CBF_TASK_KDE, tMax, nPts, h, amountOfInitialConditions, initialConditions,
                 ranges, indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks, transientTime,
                 values, amountOfValues, preScaller, in_kdeSampling, in_kdeSamplesInterval1,
                 in_kdeSamplesInterval2, in_kdeSamplesSmooth, 0.0, false, 6);
}

// hostLibrary.cu:1094-1266: header at default precision (:1172-1176)
void bifurcation2DDBSCANIC(const double tMax, const int nPts, const double h,
                           const int amountOfInitialConditions, const double* initialConditions,
                           const double* ranges, const int* indicesOfMutVars,
                           const int writableVar, const double maxValue,
                           const int maxAmountOfPeaks, const double transientTime,
                           const double* values, const int amountOfValues,
                           const int preScaller, const double eps)
{
    map2d_common(true, CBF_TASK_DBSCAN, tMax, nPts, h, amountOfInitialConditions,
                 initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                 maxAmountOfPeaks, transientTime, values, amountOfValues, preScaller, 0, 0.0, 0.0,
                 0.0, eps, true, 6);
}

// hostLibrary.cu:1270-1393
void LLE1D(const double tMax, const double NT, const int nPts, const double h, const double eps,
           const double* initialConditions, const int amountOfInitialConditions,
           const double* ranges, const int* indicesOfMutVars, const int writableVar,
           const double maxValue, const double transientTime, const double* values,
           const int amountOfValues)
{
    lle_common(0, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
               indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

// hostLibrary.cu:1397-1520
void LLE1DIC(const double tMax, const double NT, const int nPts, const double h, const double eps,
             const double* initialConditions, const int amountOfInitialConditions,
             const double* ranges, const int* indicesOfMutVars, const int writableVar,
             const double maxValue, const double transientTime, const double* values,
             const int amountOfValues)
{
    lle_common(1, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
               indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

// hostLibrary.cu:1524-1663
void LLE2D(const double tMax, const double NT, const int nPts, const double h, const double eps,
           const double* initialConditions, const int amountOfInitialConditions,
           const double* ranges, const int* indicesOfMutVars, const int writableVar,
           const double maxValue, const double transientTime, const double* values,
           const int amountOfValues)
{
    lle_common(2, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
               indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

// hostLibrary.cu:1666-1798
void LLE2DIC(const double tMax, const double NT, const int nPts, const double h, const double eps,
             const double* initialConditions, const int amountOfInitialConditions,
             const double* ranges, const int* indicesOfMutVars, const int writableVar,
             const double maxValue, const double transientTime, const double* values,
             const int amountOfValues)
{
    lle_common(3, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
               indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

// hostLibrary.cu:162-239: "h*j, value" rows at precision 12 (:224-233)
void modelingOneSystemDenis(const double tMax, const double h, const double hSpecial,
                            const int amountOfInitialConditions, const double* initialConditions,
                            const int writableVar, const double* values, const int amountOfValues)
{
    const double nd = (h != 0) ? tMax / h : 0.0;
    const long long n = (nd > 0 && nd < 2147483648.0) ? (long long)(int)nd : 0;
    std::vector<double> res((size_t)n);
    CBF_CHECK(cbf_modeling_one_system(current_system(), tMax, h, hSpecial, amountOfInitialConditions,
                                      initialConditions, writableVar, values, amountOfValues, res.data(),
                                      n));
    CsvOut out(current_path());
    out.precision(12);
    if (n > 0 && !out.is_open()) io_check(CBF_ERR_IO);
    for (long long j = 0; j < n; ++j) {
        out.dbl(h * (double)(size_t)j);
        out.str(", ");
        out.dbl(res[(size_t)j]);
        out.str("\n");
    }
}

// hostLibrary.cu:748-925: header and values at the default precision (:805-809, :887-902)
void calculationOfPeriodicityByOstrovsky(const double tMax, const int nPts, const double h,
                                         const int amountOfInitialConditions,
                                         const double* initialConditions, const double* ranges,
                                         const int* indicesOfMutVars, const int writableVar,
                                         const double maxValue, const int maxAmountOfPeaks,
                                         const double transientTime, const double* values,
                                         const int amountOfValues, const int preScaller,
                                         const double eps, const double ostrovskyThreshold)
{
    std::vector<double> res((size_t)nPts * (size_t)nPts);
    CBF_CHECK(cbf_ostrovsky2d(current_system(), tMax, nPts, h, amountOfInitialConditions, initialConditions,
                              ranges, indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks,
                              transientTime, values, amountOfValues, preScaller, eps, ostrovskyThreshold,
                              res.data()));
    io_check(cbf_csv_write_map(current_path().c_str(), res.data(), 1, (int64_t)res.size(), nPts, ranges, 6));
}

// hostLibrary.cu:1802-1924
void LS1D(const double tMax, const double NT, const int nPts, const double h, const double eps,
          const double* initialConditions, const int amountOfInitialConditions,
          const double* ranges, const int* indicesOfMutVars, const int writableVar,
          const double maxValue, const double transientTime, const double* values,
          const int amountOfValues)
{
    ls_common(1, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
              indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

// hostLibrary.cu:1928-2082
void LS2D(const double tMax, const double NT, const int nPts, const double h, const double eps,
          const double* initialConditions, const int amountOfInitialConditions,
          const double* ranges, const int* indicesOfMutVars, const int writableVar,
          const double maxValue, const double transientTime, const double* values,
          const int amountOfValues)
{
    ls_common(2, tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
              indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues);
}

void cbfSetSystem(int system) { g_system.store(system); }
int cbfGetSystem() { return current_system(); }
void cbfSetSurrogate(int enable) { g_surrogate.store(enable < 0 ? -1 : (enable ? 1 : 0)); }
int cbfGetSurrogate() { return surrogate_enabled() ? 1 : 0; }

void cbfSetOutputPath(const char* path)
{
    std::lock_guard<std::mutex> lk(g_path_mu);
    if (path) {
        g_path = path;
        g_path_set = true;
    } else {
        g_path.clear();
        g_path_set = false;
    }
}

const char* cbfGetOutputPath()
{
    static thread_local std::string s;
    s = current_path();
    return s.c_str();
}

// ---------------------------------------------------------------------------
// CSV writers with the reference's byte layout, for C-ABI callers (cbf.h).

namespace {
cbf_status open_or_fail(CsvOut& out, long long nValues)
{
    if (nValues > 0 && !out.is_open()) return CBF_ERR_IO;
    return CBF_OK;
}
}  // namespace

// NumPy .npy (format 1.0): magic, version, little-endian header length, a
// Python dict literal padded with spaces to a 64-byte boundary, then the data.
extern "C" cbf_status cbf_npy_write(const char* path, const void* values, int32_t isDouble,
                                    int64_t rows, int64_t cols)
{
    if (!path || rows < 0 || cols < 0 || (rows * cols > 0 && !values)) return CBF_ERR_INVALID_ARG;
    char dict[160];
    int len = snprintf(dict, sizeof(dict), "{'descr': '%s', 'fortran_order': False, 'shape': (%lld, %lld), }",
                       isDouble ? "<f8" : "<i4", (long long)rows, (long long)cols);
    std::string hdr(dict, (size_t)len);
    const size_t pre = 10;  // magic (6) + version (2) + length (2)
    while ((pre + hdr.size() + 1) % 64 != 0) hdr.push_back(' ');
    hdr.push_back('\n');
    FILE* f = fopen(path, "wb");
    if (!f) return CBF_ERR_IO;
    const unsigned char head[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(hdr.size() & 0xff),
                                    (unsigned char)(hdr.size() >> 8)};
    const size_t bytes = (size_t)(rows * cols) * (isDouble ? sizeof(double) : sizeof(int32_t));
    bool ok = fwrite(head, 1, 10, f) == 10 && fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() &&
              (bytes == 0 || fwrite(values, 1, bytes, f) == bytes);
    ok = (fclose(f) == 0) && ok;
    return ok ? CBF_OK : CBF_ERR_IO;
}

extern "C" cbf_status cbf_csv_write_map(const char* path, const void* values, int32_t isDouble,
                                        int64_t n, int32_t nPts, const double* headerRanges,
                                        int32_t precision)
{
    if (!path || (n > 0 && !values) || nPts < 1) return CBF_ERR_INVALID_ARG;
    CsvOut out(path);
    out.precision(precision);
    if (headerRanges) write_header(out, headerRanges);
    if (open_or_fail(out, n) != CBF_OK) return CBF_ERR_IO;
    if (isDouble)
        write_map_parallel(out, (const double*)values, n, nPts);
    else
        write_map_parallel(out, (const int32_t*)values, n, nPts);
    // optional binary copy of the map beside the CSV (rows of nPts values)
    const char* side = getenv("CBF_NPY_SIDECAR");
    if (side && *side && strcmp(side, "0") != 0) {
        const std::string np = std::string(path) + ".npy";
        const long long rows = (n + nPts - 1) / nPts;
        if (rows * nPts == n) return cbf_npy_write(np.c_str(), values, isDouble, rows, nPts);
        return cbf_npy_write(np.c_str(), values, isDouble, 1, n);
    }
    return CBF_OK;
}

extern "C" cbf_status cbf_csv_write_peaks(const char* path, int32_t nPts, const double* ranges,
                                          int64_t firstPoint, int64_t nPoints, const double* peaks,
                                          int32_t peakCapacity, const int32_t* counts,
                                          int32_t append)
{
    if (!path || !ranges || (nPoints > 0 && (!peaks || !counts))) return CBF_ERR_INVALID_ARG;
    CsvOut out(path, append != 0);
    out.precision(12);  // hostLibrary.cu:125
    long long total = 0;
    for (long long k = 0; k < nPoints; ++k) total += counts[k];
    if (open_or_fail(out, total) != CBF_OK) return CBF_ERR_IO;
    // "param, peak\n" per peak (hostLibrary.cu:127-138)
    for (long long k = 0; k < nPoints; ++k) {
        const double param = host_value_by_idx((int)(firstPoint + k), nPts, ranges[0], ranges[1], 0);
        for (int j = 0; j < counts[k]; ++j) {
            out.dbl(param);
            out.str(", ");
            out.dbl(peaks[(size_t)k * peakCapacity + j]);
            out.str("\n");
        }
    }
    return CBF_OK;
}

extern "C" cbf_status cbf_csv_write_pairs(const char* path, int32_t nPts, const double* ranges,
                                          const double* values, int64_t n, int32_t precision)
{
    if (!path || !ranges || (n > 0 && !values)) return CBF_ERR_INVALID_ARG;
    CsvOut out(path);
    out.precision(precision);
    if (open_or_fail(out, n) != CBF_OK) return CBF_ERR_IO;
    // "param, value\n" (hostLibrary.cu:1368-1378)
    for (long long k = 0; k < n; ++k) {
        out.dbl(host_value_by_idx((int)k, nPts, ranges[0], ranges[1], 0));
        out.str(", ");
        out.dbl(values[k]);
        out.str("\n");
    }
    return CBF_OK;
}

extern "C" cbf_status cbf_csv_write_rows(const char* path, int32_t nPts, const double* ranges,
                                         const double* values, int64_t n, int32_t nCols,
                                         int32_t precision)
{
    if (!path || !ranges || nCols < 0 || (n > 0 && nCols > 0 && !values)) return CBF_ERR_INVALID_ARG;
    CsvOut out(path);
    out.precision(precision);
    if (open_or_fail(out, n) != CBF_OK) return CBF_ERR_IO;
    // "param, v1, ..., vN\n" (hostLibrary.cu:1900-1910)
    for (long long k = 0; k < n; ++k) {
        out.dbl(host_value_by_idx((int)k, nPts, ranges[0], ranges[1], 0));
        for (int c = 0; c < nCols; ++c) {
            out.str(", ");
            out.dbl(values[(size_t)k * nCols + c]);
        }
        out.str("\n");
    }
    return CBF_OK;
}

// C-callable access to the facade for bindings without C++ name mangling
// (ctypes, cgo): same arguments as the C++ functions above.
extern "C" {
void cbf_facade_set_system(int system) { cbfSetSystem(system); }
void cbf_facade_set_output_path(const char* path) { cbfSetOutputPath(path); }
void cbf_facade_set_surrogate(int enable) { cbfSetSurrogate(enable); }
}
