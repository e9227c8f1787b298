// host.cpp -- host side of libctc: errors, tensor I/O, sorting, the CISS
// builder, reference lane multiplicities, work-tile planning, factor models.
#include "ctc_internal.h"

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <charconv>
#include <condition_variable>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <numeric>
#include <parallel/algorithm>
#include <thread>

namespace ctc {

static thread_local std::string g_last_error;

void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

void fail(int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Error(code, buf);
}

int host_threads()
{
    static int n = [] {
        const char *e = getenv("CTC_HOST_THREADS");
        int v = e ? atoi(e) : (int)std::thread::hardware_concurrency();
        return v < 1 ? 1 : (v > 64 ? 64 : v);
    }();
    return n;
}

// Persistent host workers (host_threads() - 1 of them; the calling thread
// works too): parallel loops over staging chunks no longer create and join
// a thread set per call.  One job runs at a time; callers from several
// threads queue on run_mu, and a loop started inside a task runs inline.
// A task that throws (an allocation failure, a library error) does not end
// the process: the job's other tasks still run, and the first exception is
// rethrown to the caller once all of them are done.
namespace {
thread_local bool tl_in_task = false;

struct HostPool {
    std::mutex run_mu, mu;
    std::condition_variable cv_start, cv_done;
    const std::function<void(int)> *job = nullptr;
    std::exception_ptr err;
    int ntasks = 0, next = 0, pending = 0;
    uint64_t gen = 0;
    bool stop = false;
    std::vector<std::thread> workers;

    explicit HostPool(int nworkers)
    {
        for (int i = 0; i < nworkers; ++i) workers.emplace_back([this] { loop(); });
    }
    ~HostPool()
    {
        {
            std::lock_guard<std::mutex> l(mu);
            stop = true;
        }
        cv_start.notify_all();
        for (auto &t : workers) t.join();
    }
    // take tasks of the current job until none is left (mu held on entry and exit)
    void drain(std::unique_lock<std::mutex> &l)
    {
        while (next < ntasks) {
            const int t = next++;
            const std::function<void(int)> *f = job;
            l.unlock();
            tl_in_task = true;
            std::exception_ptr e;
            try {
                (*f)(t);
            } catch (...) {
                e = std::current_exception();
            }
            tl_in_task = false;
            l.lock();
            if (e && !err) err = e;
            if (--pending == 0) cv_done.notify_all();
        }
    }
    void loop()
    {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> l(mu);
        for (;;) {
            cv_start.wait(l, [&] { return stop || gen != seen; });
            if (stop) return;
            seen = gen;
            drain(l);
        }
    }
    void run(int n, const std::function<void(int)> &f)
    {
        std::lock_guard<std::mutex> g(run_mu);
        std::unique_lock<std::mutex> l(mu);
        job = &f;
        ntasks = n;
        next = 0;
        pending = n;
        ++gen;
        cv_start.notify_all();
        drain(l);
        cv_done.wait(l, [&] { return pending == 0; });
        job = nullptr;
        std::exception_ptr e = err;
        err = nullptr;
        if (e) std::rethrow_exception(e);
    }
};
}  // namespace

void host_run(int ntasks, const std::function<void(int)> &task)
{
    static HostPool pool(host_threads() - 1);
    if (ntasks <= 1 || host_threads() == 1 || tl_in_task) {
        for (int t = 0; t < ntasks; ++t) task(t);
        return;
    }
    pool.run(ntasks, task);
}

template <typename F>
static void parallel_for(uint64_t n, F &&fn)
{
    int P = host_threads();
    if (n < 65536 || P == 1) {
        fn(0, 0, n);
        return;
    }
    const std::function<void(int)> task = [&](int p) { fn(p, n * p / P, n * (p + 1) / P); };
    host_run(P, task);
}

// ------------------------------------------------------------------
// .tns text reader
// ------------------------------------------------------------------

// Token parsers with strtoul / strtod semantics.  The common form
// (optional blanks, plain decimal digits, a separator or the line end after
// the token) goes through std::from_chars, which is correctly rounded like
// glibc's strtod and several times faster; anything else (a sign, a hex
// float, a token glued to other text) is handed to strtoul / strtod
// unchanged, so every input parses as the reference's reader parses it.
static inline bool token_end(const char *p, const char *end)
{
    return p >= end || *p == ' ' || *p == '\t' || *p == '\r' || *p == '\0';
}

static inline uint64_t parse_index(char *&ptr, const char *end)
{
    const char *q = ptr;
    while (q < end && (*q == ' ' || *q == '\t')) ++q;
    uint64_t v = 0;
    const auto r = std::from_chars(q, end, v, 10);
    if (r.ec == std::errc() && token_end(r.ptr, end)) {
        ptr = const_cast<char *>(r.ptr);
        return v;
    }
    return strtoul(ptr, &ptr, 10);
}

static inline double parse_value(char *&ptr, const char *end)
{
    const char *q = ptr;
    while (q < end && (*q == ' ' || *q == '\t')) ++q;
    // digits only (inf / nan spellings and their NaN payloads stay strtod's)
    const char *d = (q < end && *q == '-') ? q + 1 : q;
    if (d >= end || !((*d >= '0' && *d <= '9') || *d == '.')) return strtod(ptr, &ptr);
    double v = 0;
    const auto r = std::from_chars(q, end, v);
    if (r.ec == std::errc() && token_end(r.ptr, end)) {
        ptr = const_cast<char *>(r.ptr);
        return v;
    }
    return strtod(ptr, &ptr);
}

// Restates sgpu/io.c:234-308 (tt_get_dims) + io.c:58-106 (p_tt_read_file):
// the mode count comes from the first data line split on " \t" (the value
// token and the trailing newline token excluded), a data line is one whose
// getline() length exceeds 1 and that does not start with '#', indices are
// strtoul base 10 (kept as read), values strtod.  The file is parsed in
// parallel over line-aligned chunks.
static void read_tns(const char *path, ctc_tensor &t)
{
    const int fd = open(path, O_RDONLY);
    if (fd < 0) fail(CTC_E_IO, "cannot open '%s'", path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        fail(CTC_E_IO, "cannot stat '%s'", path);
    }
    const size_t N = (size_t)st.st_size;
    // an uninitialised buffer, read by byte ranges on the host threads
    std::unique_ptr<char[]> buf(new char[N + 1]);
    char *data = buf.get();
    {
        const int RP = N < ((size_t)8 << 20) ? 1 : host_threads();
        std::atomic<int> short_read{0};
        const std::function<void(int)> rd = [&](int p) {
            size_t b = N * (size_t)p / RP;
            const size_t e = N * (size_t)(p + 1) / RP;
            while (b < e) {
                const ssize_t r = pread(fd, data + b, e - b, (off_t)b);
                if (r <= 0) {
                    short_read = 1;
                    return;
                }
                b += (size_t)r;
            }
        };
        host_run(RP, rd);
        close(fd);
        if (short_read) fail(CTC_E_IO, "short read on '%s'", path);
    }
    data[N] = '\0';

    // mode count from the first data line (reference counts strtok tokens
    // on " \t", where the last token carries the newline, then subtracts 1)
    int nmodes = -1;
    {
        size_t p = 0;
        while (p < N) {
            size_t e = p;
            while (e < N && data[e] != '\n') ++e;
            size_t len = e - p + (e < N ? 1 : 0);
            if (len > 1 && data[p] != '#') {
                std::string line(data + p, data + e + (e < N ? 1 : 0));
                int ntok = 0;
                char *save = nullptr;
                for (char *tok = strtok_r(&line[0], " \t", &save); tok;
                     tok = strtok_r(nullptr, " \t", &save))
                    ++ntok;
                nmodes = ntok - 1;
                break;
            }
            p = e + 1;
        }
    }
    if (nmodes < 1 || nmodes > 4) fail(CTC_E_IO, "'%s': cannot determine the number of modes", path);

    // line-aligned chunks
    int P = host_threads();
    if (N < (1u << 20)) P = 1;
    std::vector<size_t> cut(P + 1, 0);
    cut[P] = N;
    for (int p = 1; p < P; ++p) {
        size_t c = N * p / P;
        while (c < N && data[c - 1] != '\n') ++c;
        cut[p] = std::max(c, cut[p - 1]);
    }
    auto is_data = [&](size_t p, size_t e) {
        size_t len = e - p + (e < N ? 1 : 0);
        return len > 1 && data[p] != '#';
    };
    // count the data lines of each chunk, NUL-terminating its lines on the
    // way so a short line cannot run into the next one
    std::vector<uint64_t> count(P, 0);
    std::vector<std::thread> th;
    for (int p = 0; p < P; ++p)
        th.emplace_back([&, p] {
            uint64_t c = 0;
            size_t q = cut[p];
            while (q < cut[p + 1]) {
                size_t e = q;
                while (e < N && data[e] != '\n' && data[e] != '\0') ++e;
                if (e < N) data[e] = '\0';
                if (is_data(q, e)) ++c;
                q = e + 1;
            }
            count[p] = c;
        });
    for (auto &x : th) x.join();
    th.clear();
    std::vector<uint64_t> off(P + 1, 0);
    for (int p = 0; p < P; ++p) off[p + 1] = off[p] + count[p];
    const uint64_t nnz = off[P];

    t.nmodes = nmodes;
    t.nnz = nnz;
    for (int m = 0; m < nmodes; ++m) t.ind[m].assign(nnz, 0);
    t.vals.assign(nnz, 0.0);
    std::vector<uint64_t> mx((size_t)P * 4, 0), mn((size_t)P * 4, 1);
    for (int p = 0; p < P; ++p)
        th.emplace_back([&, p] {
            uint64_t n = off[p];
            size_t q = cut[p];
            while (q < cut[p + 1]) {
                size_t e = q;
                while (e < N && data[e] != '\0') ++e;
                if (is_data(q, e)) {
                    char *ptr = data + q;
                    const char *end = data + e;
                    for (int m = 0; m < nmodes; ++m) {
                        uint64_t v = parse_index(ptr, end);
                        t.ind[m][n] = v;
                        if (v > mx[p * 4 + m]) mx[p * 4 + m] = v;
                        if (v < mn[p * 4 + m]) mn[p * 4 + m] = v;
                    }
                    t.vals[n] = parse_value(ptr, end);
                    ++n;
                }
                q = e + 1;
            }
        });
    for (auto &x : th) x.join();
    for (int m = 0; m < nmodes; ++m) {
        uint64_t d = 0, o = 1;
        for (int p = 0; p < P; ++p) {
            d = std::max(d, mx[p * 4 + m]);
            o = std::min(o, mn[p * 4 + m]);
        }
        t.dims[m] = d + (o == 0 ? 1 : 0);
    }
}

static const char kMagic[4] = {'C', 'T', 'C', 'B'};

// Reads `bytes` bytes at offset `off` of `fd` into dst, by byte ranges on
// the host threads; false on a short read.
static bool pread_parallel(int fd, char *dst, uint64_t bytes, off_t off)
{
    const int P = bytes < ((uint64_t)4 << 20) ? 1 : host_threads();
    std::atomic<int> short_read{0};
    const std::function<void(int)> rd = [&](int q) {
        uint64_t b = bytes * (uint64_t)q / P;
        const uint64_t e = bytes * (uint64_t)(q + 1) / P;
        while (b < e) {
            const ssize_t r = pread(fd, dst + b, e - b, off + (off_t)b);
            if (r <= 0) {
                short_read = 1;
                return;
            }
            b += (uint64_t)r;
        }
    };
    host_run(P, rd);
    return !short_read;
}

// True when `nnz` records of `per_nnz` bytes fit in the file after `off0`
// (checked before anything is sized from the header's nnz).
static bool fits_file(int fd, uint64_t off0, uint64_t nnz, uint64_t per_nnz)
{
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size < 0 || (uint64_t)st.st_size < off0) return false;
    return nnz <= ((uint64_t)st.st_size - off0) / per_nnz;
}

static void read_bin(const char *path, ctc_tensor &t)
{
    FILE *f = fopen(path, "rb");
    if (!f) fail(CTC_E_IO, "cannot open '%s'", path);
    char mg[4];
    uint32_t ver = 0, nm = 0;
    uint64_t nnz = 0;
    bool ok = fread(mg, 1, 4, f) == 4 && memcmp(mg, kMagic, 4) == 0 &&
              fread(&ver, 4, 1, f) == 1 && ver == 1 && fread(&nm, 4, 1, f) == 1 &&
              nm >= 1 && nm <= 4 && fread(&nnz, 8, 1, f) == 1;
    if (ok) ok = fread(t.dims, 8, nm, f) == nm;
    const off_t off0 = (off_t)(4 + 4 + 4 + 8 + 8 * (uint64_t)nm);
    const int fd = fileno(f);
    // the arrays must be in the file before the header's nnz sizes anything
    if (ok) ok = fits_file(fd, (uint64_t)off0, nnz, 8 * ((uint64_t)nm + 1));
    if (ok) {
        t.nmodes = (int)nm;
        t.nnz = nnz;
        const uint64_t bytes = nnz * 8;
        for (uint32_t m = 0; ok && m < nm; ++m) {
            t.ind[m].resize(nnz);
            ok = pread_parallel(fd, reinterpret_cast<char *>(t.ind[m].data()), bytes, off0 + (off_t)(m * bytes));
        }
        if (ok) {
            t.vals.resize(nnz);
            ok = pread_parallel(fd, reinterpret_cast<char *>(t.vals.data()), bytes, off0 + (off_t)(nm * bytes));
        }
    }
    fclose(f);
    if (!ok) fail(CTC_E_IO, "'%s' is not a valid CTCB tensor file", path);
}

// SPLATT coordinate binary form, as the reference writes it
// (sgpu/io.c:116-150 p_write_tt_binary_header, io.c:347-431
// tt_write_binary_file): int32 magic 0 (SPLATT_BIN_COORD, sgpu/io.h:67-84),
// u64 idx_width, u64 val_width, then idx_width-byte words: nmodes,
// dims[nmodes], nnz, the nmodes index arrays, and nnz values of val_width
// bytes.  The reference's reader (io.c:160-188, 436-509) exits on its own
// files (idx_width 8 > 4) and reads narrow indices with an uninitialised
// count; here idx_width 4 or 8 and val_width 4 or 8 are all read, indices
// kept as stored (1-based from .tns files), dims as in the header.
static void read_splatt_bin(const char *path, ctc_tensor &t)
{
    FILE *f = fopen(path, "rb");
    if (!f) fail(CTC_E_IO, "cannot open '%s'", path);
    int32_t magic = -1;
    uint64_t iw = 0, vw = 0;
    bool ok = fread(&magic, 4, 1, f) == 1 && magic == 0 && fread(&iw, 8, 1, f) == 1 && fread(&vw, 8, 1, f) == 1 &&
              (iw == 4 || iw == 8) && (vw == 4 || vw == 8);
    auto word = [&](uint64_t *v) {
        if (iw == 8) return fread(v, 8, 1, f) == 1;
        uint32_t w = 0;
        const bool r = fread(&w, 4, 1, f) == 1;
        *v = w;
        return r;
    };
    uint64_t nm = 0, nnz = 0;
    if (ok) ok = word(&nm) && nm >= 1 && nm <= 4;
    for (uint64_t m = 0; ok && m < nm; ++m) ok = word(&t.dims[m]);
    if (ok) ok = word(&nnz);
    const uint64_t off0 = 4 + 8 + 8 + iw * (nm + 2);
    const int fd = fileno(f);
    if (ok) ok = fits_file(fd, off0, nnz, iw * nm + vw);
    if (ok) {
        t.nmodes = (int)nm;
        t.nnz = nnz;
        std::vector<uint32_t, NoInitAlloc<uint32_t>> narrow;
        std::vector<float, NoInitAlloc<float>> fvals;
        const uint64_t ib = nnz * iw;
        for (uint64_t m = 0; ok && m < nm; ++m) {
            t.ind[m].resize(nnz);
            const off_t at = (off_t)(off0 + m * ib);
            if (iw == 8) {
                ok = pread_parallel(fd, reinterpret_cast<char *>(t.ind[m].data()), ib, at);
            } else {
                narrow.resize(nnz);
                ok = pread_parallel(fd, reinterpret_cast<char *>(narrow.data()), ib, at);
                uint64_t *dst = t.ind[m].data();
                parallel_for(nnz, [&](int, uint64_t b, uint64_t e) {
                    for (uint64_t i = b; i < e; ++i) dst[i] = narrow[i];
                });
            }
        }
        if (ok) {
            t.vals.resize(nnz);
            const off_t at = (off_t)(off0 + nm * ib);
            if (vw == 8) {
                ok = pread_parallel(fd, reinterpret_cast<char *>(t.vals.data()), nnz * 8, at);
            } else {
                fvals.resize(nnz);
                ok = pread_parallel(fd, reinterpret_cast<char *>(fvals.data()), nnz * 4, at);
                double *dst = t.vals.data();
                parallel_for(nnz, [&](int, uint64_t b, uint64_t e) {
                    for (uint64_t i = b; i < e; ++i) dst[i] = (double)fvals[i];
                });
            }
        }
    }
    fclose(f);
    if (!ok) fail(CTC_E_IO, "'%s' is not a valid SPLATT binary coordinate tensor", path);
}

// ------------------------------------------------------------------
// CISS builder
// ------------------------------------------------------------------

// The value store of the reference CISS goes through an idx_t
// (sgpu/ciss.c:163 "tmpv = newtensor->vals[m]"): restated as the x86-64
// conversion sequence (signed truncation below 2^63, offset + bit flip
// above, 0x8000000000000000 for NaN and out-of-range).
static uint64_t value_through_idx(double v)
{
    const double two63 = 9223372036854775808.0;
    if (std::isnan(v)) return 0x8000000000000000ULL;
    if (v < two63) {
        if (v < -two63) return 0x8000000000000000ULL;
        return (uint64_t)(int64_t)v;
    }
    double w = v - two63;
    uint64_t r = (w < two63) ? (uint64_t)(int64_t)w : 0x8000000000000000ULL;
    return r ^ 0x8000000000000000ULL;
}

}  // namespace ctc

double ctc_value_through_idx(double v) { return (double)ctc::value_through_idx(v); }

namespace ctc {

// sgpu/ciss.c:68-195 / ga/ciss.c:69-212 with a runtime tile length.
static void build_ciss(const ctc_tensor &t, int mode, int T, bool ga, ctc_ciss &c)
{
    if (t.nmodes != 3) fail(CTC_E_UNSUP, "CISS needs an order-3 tensor (got %d)", t.nmodes);
    if (t.nnz == 0) fail(CTC_E_ARG, "CISS of an empty tensor");
    if (T < 1 || T > 64) fail(CTC_E_ARG, "tile length %d outside [1, 64]", T);
    if (mode < 0 || mode > 2) fail(CTC_E_ARG, "mode %d outside [0, 2]", mode);
    const uint64_t nnz = t.nnz;
    const uint64_t *im = t.ind[mode].data();
    const uint64_t *ij = t.ind[(mode + 1) % 3].data();
    const uint64_t *ik = t.ind[(mode + 2) % 3].data();
    const double *vals = t.vals.data();
    c.nnz = nnz;
    c.tile_len = T;
    const uint64_t ntiles = nnz / (uint64_t)T + 1;  // the last one holds the terminator
    c.size_rows = ntiles + nnz + 1;
    const uint64_t cap = c.size_rows * 3;
    // The reference loop (ciss.c:89-195) is sequential, but a tile depends on
    // the tiles before it only through the directory index of the row of the
    // nonzero just before it.  Chunks of whole tiles therefore run that loop
    // in parallel once a first pass has counted each chunk's row changes;
    // with one chunk it is the reference loop itself.
    int P = host_threads();
    if (nnz < ((uint64_t)1 << 18)) P = 1;
    if ((uint64_t)P > ntiles) P = (int)ntiles;
    std::vector<uint64_t> tb(P + 1), mb(P + 1), changes(P, 0), base(P + 1, 0);
    for (int q = 0; q <= P; ++q) {
        tb[q] = ntiles * (uint64_t)q / (uint64_t)P;
        mb[q] = q == P ? nnz : std::min<uint64_t>(tb[q] * (uint64_t)T, nnz);
    }
    const std::function<void(int)> count = [&](int q) {
        uint64_t k = 0;
        for (uint64_t m = std::max<uint64_t>(mb[q], 1); m < mb[q + 1]; ++m) k += im[m] != im[m - 1];
        changes[q] = k;
    };
    host_run(P, count);
    for (int q = 0; q < P; ++q) base[q + 1] = base[q] + changes[q];
    // directory: distinct mode indices in order of appearance (ciss.c:89-115);
    // dcounter[0] = 0 and dcounter[k] = start(slice k) - 1, the inclusive end
    // of slice k-1, which is what the reference's running counter
    // (ciss.c:97-114) accumulates; the last slot is nnz-1 (ciss.c:110).
    // ga/ciss.c:101-120 starts its running count at the first nonzero, so
    // there the counters are one larger: dcounter[k] = start(slice k).
    c.dlength = 1 + base[P];
    c.directory.assign(c.dlength, 0);
    c.dcounter.assign(c.dlength + 1, 0);
    c.directory[0] = im[0];
    const std::function<void(int)> fill_dir = [&](int q) {
        uint64_t k = base[q];
        for (uint64_t m = std::max<uint64_t>(mb[q], 1); m < mb[q + 1]; ++m)
            if (im[m] != im[m - 1]) {
                ++k;
                c.directory[k] = im[m];
                c.dcounter[k] = ga ? m : m - 1;
            }
    };
    host_run(P, fill_dir);
    c.dcounter[c.dlength] = nnz - 1;
    const uint64_t *dir = c.directory.data();
    c.entries.resize(cap);
    c.written.resize(cap);
    double *E = c.entries.data();
    uint8_t *Wr = c.written.data();
    std::atomic<int> overflow{0};
    const uint64_t row3 = ((uint64_t)T + 1) * 3;
    const std::function<void(int)> tiles = [&](int q) {
        // this chunk's tile rows start zeroed (slots the loop leaves unwritten
        // stay 0); the last chunk also clears the unused tail
        const uint64_t z0 = std::min(tb[q] * row3, cap);
        const uint64_t z1 = q == P - 1 ? cap : std::min(tb[q + 1] * row3, cap);
        std::fill(E + z0, E + z1, 0.0);
        std::fill(Wr + z0, Wr + z1, (uint8_t)0);
        uint64_t m = mb[q];
        uint64_t nl = m == 0 ? 0 : base[q];  // directory index of the row of nonzero m - 1
        uint64_t npos = tb[q] * row3;
        const uint64_t mend = q == P - 1 ? nnz + 1 : mb[q + 1];
        bool bad = false;
        auto put = [&](uint64_t off, double v) {
            const uint64_t o = npos + off;
            if (o >= cap) {
                bad = true;
                return;
            }
            E[o] = v;
            Wr[o] = 1;
        };
        while (m < mend) {
            uint64_t bitmap = 1;
            uint64_t ns = nl;
            uint64_t niv = dir[ns];
            uint64_t lc = 1;
            put(0, -1.0 * (double)ns);
            while (lc <= (uint64_t)T) {
                if (m == nnz) {
                    put(lc * 3, -1.0);
                    put(lc * 3 + 1, -1.0);
                    put(lc * 3 + 2, -1.0);
                    m++;
                    break;
                }
                uint64_t ti = im[m];
                if (ti == niv) {
                    bitmap = (bitmap << 1) + 1;
                } else {
                    bitmap = bitmap << 1;
                    niv = ti;
                    nl++;
                    put(1, -1.0 * (double)nl);
                }
                put(lc * 3, (double)ij[m]);
                put(lc * 3 + 1, (double)ik[m]);
                put(lc * 3 + 2, (double)value_through_idx(vals[m]));
                put(2, (double)bitmap);
                m++;
                lc++;
            }
            npos += row3;
        }
        if (bad) overflow = 1;
    };
    host_run(P, tiles);
    if (overflow) fail(CTC_E_ARG, "CISS layout overflow");
}

static uint64_t brev64(uint64_t x)
{
    x = ((x >> 1) & 0x5555555555555555ULL) | ((x & 0x5555555555555555ULL) << 1);
    x = ((x >> 2) & 0x3333333333333333ULL) | ((x & 0x3333333333333333ULL) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0FULL) | ((x & 0x0F0F0F0F0F0F0F0FULL) << 4);
    x = ((x >> 8) & 0x00FF00FF00FF00FFULL) | ((x & 0x00FF00FF00FF00FFULL) << 8);
    x = ((x >> 16) & 0x0000FFFF0000FFFFULL) | ((x & 0x0000FFFF0000FFFFULL) << 16);
    return (x >> 32) | (x << 32);
}

// Multiplicity with which the reference's warp kernels (sgpu/als.cu:227-312
// for ALS, kernel 0; sgpu/ccd.cu:120-200 for CCD, kernel 1) add each
// nonzero of a 32-long CISS tile into its row: the tile's first row segment
// is never written (lane 0 has mybit forced to 1), a segment ending at lane
// 31 gets K-(31-h) extra copies of lane 31 (shfl_down there returns the
// lane's own value; K = continuation bits of the tile, h = segment head),
// and the CCD kernel's grid reaches only tiles < 8*(tilenum/256+1)
// (sgpu/ccd.cu:520).  In a partial last tile the reference reads an
// inactive lane (undefined); here the inactive lanes count as new rows.
void compat_weights(const ctc_ciss &c, int kernel, std::vector<double> &w)
{
    if (c.tile_len != 32) fail(CTC_E_ARG, "compat multiplicities need tile length 32");
    const uint64_t nnz = c.nnz, tilenum = nnz / 32 + 1;
    uint64_t covered = tilenum;
    if (kernel == 1) covered = std::min<uint64_t>(tilenum, 8 * (tilenum / 256 + 1));
    w.assign(nnz, 0.0);
    for (uint64_t tile = 0; tile < covered; ++tile) {
        const uint64_t first = tile * 32;
        if (first >= nnz) break;
        const int active = (int)std::min<uint64_t>(32, nnz - first);
        uint64_t B = (uint64_t)c.entries[tile * 33 * 3 + 2];
        if (B == 0) continue;
        uint64_t b = brev64(B);
        while ((b & 1) == 0) b >>= 1;
        b >>= 1;
        const int K = __builtin_popcountll(b) - (int)(b & 1);
        int h = -1;
        for (int l = 0; l <= active; ++l) {
            bool head = (l == active) || (l > 0 && ((b >> l) & 1) == 0);
            if (!head) continue;
            if (h >= 1) {
                int e = l - 1;
                for (int q = h; q <= e; ++q) w[first + q] = 1.0;
                if (e == 31 && h < 31) w[first + 31] += (double)(K - (31 - h));
            }
            h = l;
        }
    }
}

// ------------------------------------------------------------------
// work tiles
// ------------------------------------------------------------------
// Rows of a mode-sorted copy read straight from its 1-based index array.
// A row that is smaller than the one before it marks the copy unsorted.
struct SortedRows {
    const uint64_t *ind;
    uint64_t n;
    bool bad = false;
    uint32_t operator()(uint64_t i) const { return (uint32_t)(ind[i] - 1); }
    // end of the run of equal rows that starts at i
    uint64_t run_end(uint64_t i)
    {
        const uint64_t r = ind[i];
        uint64_t e = i + 1;
        while (e < n && ind[e] == r) ++e;
        if (e < n && ind[e] < r) bad = true;
        return e;
    }
};

static TilePlan plan_span(SortedRows rows, uint32_t T, bool *unsorted)
{
    const uint64_t n = rows.n;
    TilePlan p;
    p.tiles.reserve((size_t)(n / std::max<uint32_t>(T / 2, 1) + 16) * 4);
    uint64_t i = 0;
    while (i < n) {
        uint64_t e = rows.run_end(i);
        uint64_t len = e - i;
        if (len > T) {
            uint32_t h = p.nheavy();
            uint32_t first = p.ntiles();
            uint32_t np = (uint32_t)((len + T - 1) / T);
            for (uint32_t q = 0; q < np; ++q) {
                uint64_t s = i + (uint64_t)q * T;
                p.tiles.insert(p.tiles.end(),
                               {(int32_t)s, (int32_t)std::min<uint64_t>(T, e - s), (int32_t)h, (int32_t)q});
            }
            p.heavy_rows.insert(p.heavy_rows.end(), {rows(i), first, np, 0u});
            i = e;
            continue;
        }
        // pack whole light rows (the run found above is the first of them)
        uint64_t s = i, size = 0;
        while (i < n) {
            const uint64_t ee = (i == s) ? e : rows.run_end(i);
            const uint64_t l = ee - i;
            if (l > T || size + l > T) break;
            size += l;
            i = ee;
        }
        p.tiles.insert(p.tiles.end(), {(int32_t)s, (int32_t)size, -1, 0});
    }
    if (rows.bad) *unsorted = true;
    return p;
}

// Tiles of at most T nonzeros over a copy sorted by one mode (ind: that
// mode's 1-based indices): whole light rows packed greedily, rows longer
// than T split into pieces of T.  Built over 64 row-aligned chunks in
// parallel (the chunk count is fixed, so the plan does not depend on the
// host's core count); light tiles do not straddle a chunk boundary.
// *unsorted is set when the indices decrease anywhere.
TilePlan plan_tiles_chunked(const uint64_t *ind, uint64_t n, uint32_t T, bool *unsorted)
{
    constexpr int K = 64;
    *unsorted = false;
    const int chunks = n < ((uint64_t)1 << 20) ? 1 : K;
    std::vector<uint64_t> cut(chunks + 1, 0);
    cut[chunks] = n;
    for (int c = 1; c < chunks; ++c) {
        uint64_t x = std::max<uint64_t>(n * (uint64_t)c / chunks, cut[c - 1]);
        while (x > 0 && x < n && ind[x] == ind[x - 1]) ++x;
        cut[c] = x;
    }
    for (int c = 1; c < chunks; ++c)
        if (cut[c] > 0 && cut[c] < n && ind[cut[c]] < ind[cut[c] - 1]) *unsorted = true;
    std::vector<TilePlan> part(chunks);
    std::vector<char> bad(chunks, 0);
    {
        const int P = std::max(1, std::min(host_threads(), chunks));
        std::vector<std::thread> th;
        for (int q = 0; q < P; ++q)
            th.emplace_back([&, q] {
                for (int c = q; c < chunks; c += P) {
                    bool b = false;
                    part[c] = plan_span(SortedRows{ind + cut[c], cut[c + 1] - cut[c]}, T, &b);
                    bad[c] = b;
                }
            });
        for (auto &t : th) t.join();
    }
    for (char b : bad)
        if (b) *unsorted = true;
    if (chunks == 1) return std::move(part[0]);
    TilePlan p;
    size_t nt = 0, nh = 0;
    for (const TilePlan &q : part) {
        nt += q.tiles.size();
        nh += q.heavy_rows.size();
    }
    p.tiles.reserve(nt);
    p.heavy_rows.reserve(nh);
    for (int c = 0; c < chunks; ++c) {
        const uint32_t tbase = p.ntiles(), hbase = p.nheavy();
        const TilePlan &q = part[c];
        for (size_t t = 0; t < q.tiles.size(); t += 4) {
            const int32_t h = q.tiles[t + 2];
            p.tiles.insert(p.tiles.end(), {(int32_t)(q.tiles[t] + (int64_t)cut[c]), q.tiles[t + 1],
                                           h >= 0 ? h + (int32_t)hbase : h, q.tiles[t + 3]});
        }
        for (size_t h = 0; h < q.heavy_rows.size(); h += 4)
            p.heavy_rows.insert(p.heavy_rows.end(), {q.heavy_rows[h], q.heavy_rows[h + 1] + tbase,
                                                     q.heavy_rows[h + 2], q.heavy_rows[h + 3]});
    }
    return p;
}

// The plan of plan_tiles_chunked from the copy's row runs (run r: row
// rows[r] repeated counts[r] times, in order): the chunk cut c is the first
// run start at or after n*c/64 (a cut never precedes the one before it),
// light tiles end at a cut, and tiles / heavy rows are numbered in order,
// so the two builders give the same plan.  O(runs + tiles).  Rows longer
// than H (0: T) get tiles of their own, pieces of at most T nonzeros.
// The chunks are planned in parallel on the host workers (heavy-row
// numbers and first tiles counted within the chunk), then laid end to end.
static TilePlan plan_run_span(const uint32_t *rows, const uint32_t *counts, const uint64_t *start, uint64_t r,
                              uint64_t rend, uint32_t T, uint32_t H)
{
    TilePlan p;
    p.tiles.reserve((size_t)((start[rend] - start[r]) / std::max<uint32_t>(T / 2, 1) + 16) * 4);
    auto tile = [&p](uint64_t s, uint64_t len, int32_t h, int32_t q) {
        p.tiles.push_back((int32_t)s);
        p.tiles.push_back((int32_t)len);
        p.tiles.push_back(h);
        p.tiles.push_back(q);
    };
    while (r < rend) {
        const uint64_t len = counts[r];
        if (len > H) {
            const uint32_t h = p.nheavy(), first = p.ntiles();
            const uint32_t np = (uint32_t)((len + T - 1) / T);
            const uint64_t s0 = start[r], e = s0 + len;
            for (uint32_t q = 0; q < np; ++q) {
                const uint64_t s = s0 + (uint64_t)q * T;
                tile(s, std::min<uint64_t>(T, e - s), (int32_t)h, (int32_t)q);
            }
            p.heavy_rows.insert(p.heavy_rows.end(), {rows[r], first, np, 0u});
            ++r;
            continue;
        }
        const uint64_t s = start[r];
        uint64_t size = 0;
        while (r < rend) {
            const uint64_t l = counts[r];
            if (l > H || size + l > T) break;
            size += l;
            ++r;
        }
        tile(s, size, -1, 0);
    }
    return p;
}

TilePlan plan_tiles_runs(const uint32_t *rows, const uint32_t *counts, uint64_t nruns, uint32_t T, uint32_t H)
{
    if (H == 0 || H > T) H = T;
    std::vector<uint64_t> start(nruns + 1, 0);
    for (uint64_t r = 0; r < nruns; ++r) start[r + 1] = start[r] + counts[r];
    const uint64_t n = start[nruns];
    constexpr int K = 64;
    const int chunks = n < ((uint64_t)1 << 20) ? 1 : K;
    std::vector<uint64_t> cut(chunks + 1, 0);  // in runs
    cut[chunks] = nruns;
    for (int c = 1; c < chunks; ++c) {
        const uint64_t x = std::max<uint64_t>(n * (uint64_t)c / chunks, start[cut[c - 1]]);
        cut[c] = (uint64_t)(std::lower_bound(start.begin(), start.end(), x) - start.begin());
    }
    if (chunks == 1) return plan_run_span(rows, counts, start.data(), 0, nruns, T, H);
    std::vector<TilePlan> part(chunks);
    host_run(chunks, [&](int c) { part[c] = plan_run_span(rows, counts, start.data(), cut[c], cut[c + 1], T, H); });
    std::vector<uint32_t> tbase(chunks + 1, 0), hbase(chunks + 1, 0);
    for (int c = 0; c < chunks; ++c) {
        tbase[c + 1] = tbase[c] + part[c].ntiles();
        hbase[c + 1] = hbase[c] + part[c].nheavy();
    }
    TilePlan p;
    p.tiles.resize((size_t)tbase[chunks] * 4);
    p.heavy_rows.resize((size_t)hbase[chunks] * 4);
    host_run(chunks, [&](int c) {
        const TilePlan &q = part[c];
        int32_t *t = p.tiles.data() + (size_t)tbase[c] * 4;
        for (size_t i = 0; i < q.tiles.size(); i += 4) {
            const int32_t h = q.tiles[i + 2];
            t[i] = q.tiles[i];
            t[i + 1] = q.tiles[i + 1];
            t[i + 2] = h >= 0 ? h + (int32_t)hbase[c] : h;
            t[i + 3] = q.tiles[i + 3];
        }
        uint32_t *hr = p.heavy_rows.data() + (size_t)hbase[c] * 4;
        for (size_t i = 0; i < q.heavy_rows.size(); i += 4) {
            hr[i] = q.heavy_rows[i];
            hr[i + 1] = q.heavy_rows[i + 1] + tbase[c];
            hr[i + 2] = q.heavy_rows[i + 2];
            hr[i + 3] = q.heavy_rows[i + 3];
        }
    });
    return p;
}

// counter-based uniform in [0,1): splitmix64 of (seed, mode, row, col)
static inline double u01(uint64_t seed, uint64_t mode, uint64_t row, uint64_t col)
{
    uint64_t z = seed ^ (mode * 0x9E3779B97F4A7C15ULL) ^ (row * 0xBF58476D1CE4E5B9ULL) ^
                 (col * 0x94D049BB133111EBULL);
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace ctc

using namespace ctc;

// ------------------------------------------------------------------
// C ABI: errors, tensors, CISS, models
// ------------------------------------------------------------------
extern "C" const char *ctc_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *ctc_version(void) { return "ctc 0.1 (sm_100a)"; }

extern "C" int ctc_tensor_load_tns(const char *path, ctc_tensor **out)
{
    return guarded([&] {
        if (!path || !out) fail(CTC_E_ARG, "null argument");
        auto t = new ctc_tensor();
        try {
            size_t L = strlen(path);
            if (L > 5 && strcmp(path + L - 5, ".ctcb") == 0) read_bin(path, *t);
            else if (L > 4 && strcmp(path + L - 4, ".bin") == 0) read_splatt_bin(path, *t);
            else read_tns(path, *t);
        } catch (...) {
            delete t;
            throw;
        }
        *out = t;
    });
}

extern "C" int ctc_tensor_save_bin(const ctc_tensor *t, const char *path)
{
    return guarded([&] {
        if (!t || !path) fail(CTC_E_ARG, "null argument");
        FILE *f = fopen(path, "wb");
        if (!f) fail(CTC_E_IO, "cannot create '%s'", path);
        uint32_t ver = 1, nm = (uint32_t)t->nmodes;
        bool ok = fwrite(kMagic, 1, 4, f) == 4 && fwrite(&ver, 4, 1, f) == 1 &&
                  fwrite(&nm, 4, 1, f) == 1 && fwrite(&t->nnz, 8, 1, f) == 1 &&
                  fwrite(t->dims, 8, nm, f) == nm;
        for (uint32_t m = 0; ok && m < nm; ++m)
            ok = fwrite(t->ind[m].data(), 8, t->nnz, f) == t->nnz;
        if (ok) ok = fwrite(t->vals.data(), 8, t->nnz, f) == t->nnz;
        if (fclose(f) != 0) ok = false;
        if (!ok) fail(CTC_E_IO, "write to '%s' failed", path);
    });
}

extern "C" int ctc_tensor_from_coo(int nmodes, uint64_t nnz, const uint64_t *dims,
                                   const uint64_t *const *ind, const double *vals,
                                   ctc_tensor **out)
{
    return guarded([&] {
        if (nmodes < 1 || nmodes > 4 || !ind || !vals || !out) fail(CTC_E_ARG, "bad arguments");
        auto t = new ctc_tensor();
        t->nmodes = nmodes;
        t->nnz = nnz;
        for (int m = 0; m < nmodes; ++m) {
            t->ind[m].assign(ind[m], ind[m] + nnz);
            uint64_t mx = 0;
            bool zero = false;
            for (uint64_t n = 0; n < nnz; ++n) {
                mx = std::max(mx, ind[m][n]);
                zero |= ind[m][n] == 0;
            }
            t->dims[m] = dims ? dims[m] : mx + (zero ? 1 : 0);
        }
        t->vals.assign(vals, vals + nnz);
        *out = t;
    });
}

extern "C" int ctc_tensor_info(const ctc_tensor *t, int *nmodes, uint64_t *nnz, uint64_t *dims)
{
    return guarded([&] {
        if (!t) fail(CTC_E_ARG, "null tensor");
        if (nmodes) *nmodes = t->nmodes;
        if (nnz) *nnz = t->nnz;
        if (dims)
            for (int m = 0; m < t->nmodes; ++m) dims[m] = t->dims[m];
    });
}

extern "C" int ctc_tensor_export(const ctc_tensor *t, uint64_t *const *ind, double *vals)
{
    return guarded([&] {
        if (!t) fail(CTC_E_ARG, "null tensor");
        if (ind)
            for (int m = 0; m < t->nmodes; ++m)
                if (ind[m]) memcpy(ind[m], t->ind[m].data(), t->nnz * 8);
        if (vals) memcpy(vals, t->vals.data(), t->nnz * 8);
    });
}

// perm = the stable order of the pairs (k1[i], k2[i]).  When both fit one
// 64-bit key (k1 << bits(k2) | k2), a parallel LSD radix sort: per-thread
// digit histograms, offsets digit-major and thread-minor, and an in-order
// scatter of each thread's chunk keep equal keys in input order.  Small or
// wider inputs take the comparison sort.
static void stable_order(const uint64_t *k1, const uint64_t *k2, uint64_t n, std::vector<uint64_t> &perm)
{
    perm.resize(n);
    auto comparison = [&] {
        std::iota(perm.begin(), perm.end(), 0);
        __gnu_parallel::stable_sort(perm.begin(), perm.end(), [&](uint64_t a, uint64_t b) {
            return k1[a] < k1[b] || (k1[a] == k1[b] && k2[a] < k2[b]);
        });
    };
    const int P = host_threads();
    if (n < 65536 || P == 1) return comparison();
    std::vector<uint64_t> mx1(P, 0), mx2(P, 0);
    const std::function<void(int)> maxima = [&](int q) {
        uint64_t a = 0, b = 0;
        for (uint64_t i = n * q / P; i < n * (q + 1) / P; ++i) {
            a = std::max(a, k1[i]);
            b = std::max(b, k2[i]);
        }
        mx1[q] = a;
        mx2[q] = b;
    };
    host_run(P, maxima);
    auto bits = [](uint64_t v) {
        int b = 0;
        while (b < 64 && (v >> b)) ++b;
        return b;
    };
    const int b1 = bits(*std::max_element(mx1.begin(), mx1.end()));
    const int b2 = bits(*std::max_element(mx2.begin(), mx2.end()));
    const int B = b1 + b2;
    if (B > 64) return comparison();
    std::vector<uint64_t, NoInitAlloc<uint64_t>> key(n), key2(n), id2(n);  // filled before read
    uint64_t *id = perm.data();
    const std::function<void(int)> pack = [&](int q) {
        for (uint64_t i = n * q / P; i < n * (q + 1) / P; ++i) {
            key[i] = b2 == 64 ? k2[i] : ((b1 ? k1[i] << b2 : 0) | k2[i]);
            id[i] = i;
        }
    };
    host_run(P, pack);
    const int passes = (B + 11) / 12;
    const int D = passes ? (B + passes - 1) / passes : 0;
    const uint64_t NB = (uint64_t)1 << D;
    std::vector<uint64_t> hist((size_t)P * NB);
    uint64_t *src_k = key.data(), *dst_k = key2.data(), *src_i = id, *dst_i = id2.data();
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = pass * D;
        const uint64_t mask = NB - 1;
        const std::function<void(int)> histo = [&](int q) {
            uint64_t *h = hist.data() + (size_t)q * NB;
            std::fill(h, h + NB, 0);
            for (uint64_t i = n * q / P; i < n * (q + 1) / P; ++i) ++h[(src_k[i] >> shift) & mask];
        };
        host_run(P, histo);
        uint64_t run = 0;
        for (uint64_t d = 0; d < NB; ++d)
            for (int q = 0; q < P; ++q) {
                uint64_t &h = hist[(size_t)q * NB + d];
                const uint64_t c = h;
                h = run;
                run += c;
            }
        const std::function<void(int)> scatter = [&](int q) {
            uint64_t *o = hist.data() + (size_t)q * NB;
            for (uint64_t i = n * q / P; i < n * (q + 1) / P; ++i) {
                const uint64_t at = o[(src_k[i] >> shift) & mask]++;
                dst_k[at] = src_k[i];
                dst_i[at] = src_i[i];
            }
        };
        host_run(P, scatter);
        std::swap(src_k, dst_k);
        std::swap(src_i, dst_i);
    }
    if (src_i != id) std::copy(src_i, src_i + n, id);
}

extern "C" int ctc_tensor_sort(ctc_tensor *t, int mode)
{
    return guarded([&] {
        if (!t || mode < 0 || mode >= t->nmodes) fail(CTC_E_ARG, "bad sort mode");
        const uint64_t n = t->nnz;
        const uint64_t *k1 = t->ind[mode].data();
        const uint64_t *k2 = t->ind[(mode + 1) % t->nmodes].data();
        std::vector<uint64_t> perm;
        stable_order(k1, k2, n, perm);
        std::vector<uint64_t> tmp(n);
        for (int m = 0; m < t->nmodes; ++m) {
            const uint64_t *src = t->ind[m].data();
            parallel_for(n, [&](int, uint64_t b, uint64_t e) {
                for (uint64_t i = b; i < e; ++i) tmp[i] = src[perm[i]];
            });
            t->ind[m].swap(tmp);
            tmp.resize(n);
        }
        std::vector<double> tv(n);
        parallel_for(n, [&](int, uint64_t b, uint64_t e) {
            for (uint64_t i = b; i < e; ++i) tv[i] = t->vals[perm[i]];
        });
        t->vals.swap(tv);
    });
}

// ------------------------------------------------------------------
// Data preparation (software/scripts/tvtensor.py, stensor.py)
// ------------------------------------------------------------------
namespace ctc {

// MT19937 (Matsumoto and Nishimura, 1998) with the 2002 init_by_array
// seeding, as Python's `random` module uses it: random.seed(a) for an int
// a seeds with the 32-bit words of |a|, least significant first ([0] for
// 0); getrandbits(k <= 32) is the top k bits of one 32-bit output;
// randint(0, n-1) draws getrandbits(bit_length(n)) until the value is
// below n.
class PyMersenne {
    static constexpr int N = 624, M = 397;
    uint32_t mt[N];
    int mti = N + 1;

    void init_genrand(uint32_t s)
    {
        mt[0] = s;
        for (mti = 1; mti < N; ++mti) mt[mti] = 1812433253u * (mt[mti - 1] ^ (mt[mti - 1] >> 30)) + (uint32_t)mti;
    }

public:
    explicit PyMersenne(uint64_t seed)
    {
        uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        const int klen = key[1] ? 2 : 1;
        init_genrand(19650218u);
        int i = 1, j = 0;
        for (int k = std::max(N, klen); k; --k) {
            mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1664525u)) + key[j] + (uint32_t)j;
            ++i;
            ++j;
            if (i >= N) {
                mt[0] = mt[N - 1];
                i = 1;
            }
            if (j >= klen) j = 0;
        }
        for (int k = N - 1; k; --k) {
            mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1566083941u)) - (uint32_t)i;
            ++i;
            if (i >= N) {
                mt[0] = mt[N - 1];
                i = 1;
            }
        }
        mt[0] = 0x80000000u;
        mti = N;
    }

    uint32_t next()
    {
        static const uint32_t mag01[2] = {0u, 0x9908b0dfu};
        if (mti >= N) {
            int kk = 0;
            for (; kk < N - M; ++kk) {
                const uint32_t y = (mt[kk] & 0x80000000u) | (mt[kk + 1] & 0x7fffffffu);
                mt[kk] = mt[kk + M] ^ (y >> 1) ^ mag01[y & 1u];
            }
            for (; kk < N - 1; ++kk) {
                const uint32_t y = (mt[kk] & 0x80000000u) | (mt[kk + 1] & 0x7fffffffu);
                mt[kk] = mt[kk + (M - N)] ^ (y >> 1) ^ mag01[y & 1u];
            }
            const uint32_t y = (mt[N - 1] & 0x80000000u) | (mt[0] & 0x7fffffffu);
            mt[N - 1] = mt[M - 1] ^ (y >> 1) ^ mag01[y & 1u];
            mti = 0;
        }
        uint32_t y = mt[mti++];
        y ^= (y >> 11);
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= (y >> 18);
        return y;
    }

    // randint(0, n - 1) for 1 <= n <= 2^32 - 1
    uint32_t below(uint32_t n)
    {
        int k = 0;
        while (k < 32 && (n >> k)) ++k;
        for (;;) {
            const uint32_t r = next() >> (32 - k);
            if (r < n) return r;
        }
    }
};

static ctc_tensor *subset(const ctc_tensor &t, const std::vector<uint64_t> &pick)
{
    auto *o = new ctc_tensor();
    o->nmodes = t.nmodes;
    o->nnz = pick.size();
    for (int m = 0; m < t.nmodes; ++m) {
        o->ind[m].resize(pick.size());
        uint64_t mx = 0;
        bool zero = false;
        for (size_t i = 0; i < pick.size(); ++i) {
            const uint64_t v = t.ind[m][pick[i]];
            o->ind[m][i] = v;
            mx = std::max(mx, v);
            zero |= v == 0;
        }
        o->dims[m] = mx + (zero ? 1 : 0);
    }
    o->vals.resize(pick.size());
    for (size_t i = 0; i < pick.size(); ++i) o->vals[i] = t.vals[pick[i]];
    return o;
}

}  // namespace ctc

extern "C" int ctc_tensor_split(const ctc_tensor *t, uint64_t seed, ctc_tensor **train, ctc_tensor **test,
                                ctc_tensor **val)
{
    return guarded([&] {
        if (!t) fail(CTC_E_ARG, "null tensor");
        if (t->nmodes < 2) fail(CTC_E_ARG, "the split orders by the first two modes: order >= 2");
        std::vector<uint64_t> perm;
        stable_order(t->ind[0].data(), t->ind[1].data(), t->nnz, perm);
        PyMersenne rng(seed);
        std::vector<uint64_t> pick[3];
        for (uint64_t i = 0; i < t->nnz; ++i) {
            const uint32_t flag = rng.below(10);
            pick[flag < 8 ? 0 : (flag == 8 ? 1 : 2)].push_back(perm[i]);
        }
        std::unique_ptr<ctc_tensor> out[3];
        ctc_tensor **dst[3] = {train, test, val};
        for (int k = 0; k < 3; ++k)
            if (dst[k]) out[k].reset(subset(*t, pick[k]));
        for (int k = 0; k < 3; ++k)
            if (dst[k]) *dst[k] = out[k].release();
    });
}

extern "C" int ctc_tensor_write_tns(const ctc_tensor *t, const char *path, int digits)
{
    return guarded([&] {
        if (!t || !path) fail(CTC_E_ARG, "null argument");
        if (digits > 40) fail(CTC_E_ARG, "at most 40 digits after the point");
        char vfmt[16];
        if (digits < 0) snprintf(vfmt, sizeof vfmt, "%%.17g\n");
        else snprintf(vfmt, sizeof vfmt, "%%.%df\n", digits);
        FILE *f = fopen(path, "w");
        if (!f) fail(CTC_E_IO, "cannot open %s for writing", path);
        const uint64_t n = t->nnz;
        const int nm = t->nmodes;
        // blocks of lines formatted on the host threads, written in order
        const int P = host_threads();
        const uint64_t kLines = 16384;
        std::vector<std::string> out(P);
        bool ok = true;
        for (uint64_t l0 = 0; l0 < n && ok; l0 += kLines * (uint64_t)P) {
            const std::function<void(int)> fmt = [&](int q) {
                std::string &o = out[q];
                o.clear();
                const uint64_t b = std::min(n, l0 + kLines * (uint64_t)q), e = std::min(n, b + kLines);
                char buf[400];
                for (uint64_t i = b; i < e; ++i) {
                    for (int m = 0; m < nm; ++m) {
                        const int k = snprintf(buf, sizeof buf, "%llu ", (unsigned long long)t->ind[m][i]);
                        o.append(buf, (size_t)k);
                    }
                    const int k = snprintf(buf, sizeof buf, vfmt, t->vals[i]);
                    o.append(buf, (size_t)std::min<int>(k, (int)sizeof buf - 1));
                }
            };
            host_run(P, fmt);
            for (int q = 0; q < P && ok; ++q) ok = fwrite(out[q].data(), 1, out[q].size(), f) == out[q].size();
        }
        if (fclose(f) != 0) ok = false;
        if (!ok) fail(CTC_E_IO, "write to %s failed", path);
    });
}

extern "C" int ctc_tensor_save_splatt(const ctc_tensor *t, const char *path)
{
    return guarded([&] {
        if (!t || !path) fail(CTC_E_ARG, "null argument");
        const uint64_t n = t->nnz;
        const int nm = t->nmodes;
        // 4-byte words when the counts, dims and indices all fit, 4-byte
        // values when every value is exactly a float (the test the
        // reference's header writer means to make, sgpu/io.c:124-145)
        bool narrow = n <= 0xffffffffull;
        for (int m = 0; m < nm && narrow; ++m) {
            narrow = t->dims[m] <= 0xffffffffull;
            for (uint64_t i = 0; i < n && narrow; ++i) narrow = t->ind[m][i] <= 0xffffffffull;
        }
        bool fl = true;
        for (uint64_t i = 0; i < n && fl; ++i) {
            const double v = t->vals[i];
            fl = std::isnan(v) || (double)(float)v == v;
        }
        const uint64_t iw = narrow ? 4 : 8, vw = fl ? 4 : 8;
        FILE *f = fopen(path, "wb");
        if (!f) fail(CTC_E_IO, "cannot create '%s'", path);
        const int32_t magic = 0;
        bool ok = fwrite(&magic, 4, 1, f) == 1 && fwrite(&iw, 8, 1, f) == 1 && fwrite(&vw, 8, 1, f) == 1;
        auto word = [&](uint64_t v) {
            if (iw == 8) return fwrite(&v, 8, 1, f) == 1;
            const uint32_t w = (uint32_t)v;
            return fwrite(&w, 4, 1, f) == 1;
        };
        ok = ok && word((uint64_t)nm);
        for (int m = 0; m < nm && ok; ++m) ok = word(t->dims[m]);
        ok = ok && word(n);
        std::vector<uint32_t> w32;
        for (int m = 0; m < nm && ok; ++m) {
            if (iw == 8) {
                ok = fwrite(t->ind[m].data(), 8, n, f) == n;
            } else {
                w32.assign(t->ind[m].begin(), t->ind[m].end());
                ok = fwrite(w32.data(), 4, n, f) == n;
            }
        }
        if (ok) {
            if (vw == 8) {
                ok = fwrite(t->vals.data(), 8, n, f) == n;
            } else {
                std::vector<float> fv(t->vals.begin(), t->vals.end());
                ok = fwrite(fv.data(), 4, n, f) == n;
            }
        }
        if (fclose(f) != 0) ok = false;
        if (!ok) fail(CTC_E_IO, "write to '%s' failed", path);
    });
}

extern "C" int ctc_plan_tiles(const uint64_t *ind, uint64_t n, uint32_t tile_len, int from_runs, int32_t *tiles,
                              uint64_t tiles_cap, uint64_t *ntiles, uint32_t *heavy, uint64_t heavy_cap,
                              uint64_t *nheavy)
{
    return guarded([&] {
        if ((!ind && n) || !ntiles || !nheavy || tile_len == 0) fail(CTC_E_ARG, "bad arguments");
        if (n >= 0x7fffffffull) fail(CTC_E_UNSUP, "tile plans index at most 2^31 - 1 nonzeros");
        TilePlan p;
        if (from_runs) {
            std::vector<uint32_t> rows, counts;
            for (uint64_t i = 0; i < n;) {
                if (i > 0 && ind[i] < ind[i - 1]) fail(CTC_E_ARG, "indices are not sorted");
                uint64_t e = i + 1;
                while (e < n && ind[e] == ind[i]) ++e;
                rows.push_back((uint32_t)(ind[i] - 1));
                counts.push_back((uint32_t)(e - i));
                i = e;
            }
            p = plan_tiles_runs(rows.data(), counts.data(), rows.size(), tile_len);
        } else {
            bool unsorted = false;
            p = plan_tiles_chunked(ind, n, tile_len, &unsorted);
            if (unsorted) fail(CTC_E_ARG, "indices are not sorted");
        }
        *ntiles = p.ntiles();
        *nheavy = p.nheavy();
        if (tiles && tiles_cap >= p.ntiles()) std::copy(p.tiles.begin(), p.tiles.end(), tiles);
        if (heavy && heavy_cap >= p.nheavy()) std::copy(p.heavy_rows.begin(), p.heavy_rows.end(), heavy);
    });
}

extern "C" int ctc_tensor_free(ctc_tensor *t)
{
    delete t;
    return CTC_OK;
}

extern "C" int ctc_ciss_build(const ctc_tensor *t, int mode, int tile_len, ctc_ciss **out)
{
    return guarded([&] {
        if (!t || !out) fail(CTC_E_ARG, "null argument");
        auto c = new ctc_ciss();
        try {
            build_ciss(*t, mode - 1, tile_len, false, *c);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

extern "C" int ctc_ciss_build_ga(const ctc_tensor *t, int mode, int tile_len, ctc_ciss **out)
{
    return guarded([&] {
        if (!t || !out) fail(CTC_E_ARG, "null argument");
        auto c = new ctc_ciss();
        try {
            build_ciss(*t, mode - 1, tile_len, true, *c);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

extern "C" int ctc_ciss_sizes(const ctc_ciss *c, uint64_t *nnz, uint64_t *dlength,
                              uint64_t *size_rows, int *tile_len)
{
    return guarded([&] {
        if (!c) fail(CTC_E_ARG, "null CISS");
        if (nnz) *nnz = c->nnz;
        if (dlength) *dlength = c->dlength;
        if (size_rows) *size_rows = c->size_rows;
        if (tile_len) *tile_len = c->tile_len;
    });
}

extern "C" int ctc_ciss_export(const ctc_ciss *c, uint64_t *directory, uint64_t *dcounter,
                               double *entries, uint8_t *written)
{
    return guarded([&] {
        if (!c) fail(CTC_E_ARG, "null CISS");
        if (directory) memcpy(directory, c->directory.data(), c->dlength * 8);
        if (dcounter) memcpy(dcounter, c->dcounter.data(), (c->dlength + 1) * 8);
        if (entries) memcpy(entries, c->entries.data(), c->size_rows * 3 * 8);
        if (written) memcpy(written, c->written.data(), c->size_rows * 3);
    });
}

extern "C" int ctc_ciss_free(ctc_ciss *c)
{
    delete c;
    return CTC_OK;
}

extern "C" int ctc_model_create(int nmodes, const uint64_t *dims, int rank, ctc_model **out)
{
    return guarded([&] {
        if (nmodes < 1 || nmodes > 4 || !dims || rank < 1 || !out) fail(CTC_E_ARG, "bad model shape");
        auto m = new ctc_model();
        m->nmodes = nmodes;
        m->rank = rank;
        for (int q = 0; q < nmodes; ++q) {
            m->dims[q] = dims[q];
            m->U[q].assign(dims[q] * (uint64_t)rank, 0.0);
        }
        *out = m;
    });
}

extern "C" int ctc_model_init_uniform(ctc_model *m, uint64_t seed, double scale)
{
    return guarded([&] {
        if (!m) fail(CTC_E_ARG, "null model");
        for (int q = 0; q < m->nmodes; ++q) {
            const uint64_t R = (uint64_t)m->rank;
            double *U = m->U[q].data();
            parallel_for(m->dims[q], [&](int, uint64_t b, uint64_t e) {
                for (uint64_t r = b; r < e; ++r)
                    for (uint64_t f = 0; f < R; ++f) U[r * R + f] = u01(seed, (uint64_t)q, r, f) * scale;
            });
        }
    });
}

extern "C" int ctc_model_set(ctc_model *m, int mode, const double *rowmajor)
{
    return guarded([&] {
        if (!m || mode < 0 || mode >= m->nmodes || !rowmajor) fail(CTC_E_ARG, "bad argument");
        memcpy(m->U[mode].data(), rowmajor, m->U[mode].size() * 8);
    });
}

extern "C" int ctc_model_get(const ctc_model *m, int mode, double *rowmajor)
{
    return guarded([&] {
        if (!m || mode < 0 || mode >= m->nmodes || !rowmajor) fail(CTC_E_ARG, "bad argument");
        memcpy(rowmajor, m->U[mode].data(), m->U[mode].size() * 8);
    });
}

// Text form of one factor matrix, as the reference's mat_write_file
// (sgpu/io.c:565-591, row-first case): one row per line, every value
// printed "%+0.8le " (the format, with its trailing space, kept alike so
// that files compare with the reference's own output).
extern "C" int ctc_model_write_text(const ctc_model *m, int mode, const char *path)
{
    return guarded([&] {
        if (!m || mode < 0 || mode >= m->nmodes || !path) fail(CTC_E_ARG, "bad argument");
        FILE *f = fopen(path, "w");
        if (!f) fail(CTC_E_IO, "cannot open %s for writing", path);
        const double *v = m->U[mode].data();
        const uint64_t I = m->dims[mode];
        const int R = m->rank;
        // blocks of rows formatted on the host threads, written in order:
        // the same bytes as one row after another
        const int P = host_threads();
        const uint64_t kRows = 8192;
        std::vector<std::string> out(P);
        bool ok = true;
        for (uint64_t r0 = 0; r0 < I && ok; r0 += kRows * (uint64_t)P) {
            const std::function<void(int)> fmt = [&](int q) {
                std::string &o = out[q];
                o.clear();
                const uint64_t b = std::min(I, r0 + kRows * (uint64_t)q), e = std::min(I, b + kRows);
                char buf[40];
                for (uint64_t i = b; i < e; ++i) {
                    for (int j = 0; j < R; ++j) {
                        const int k = snprintf(buf, sizeof buf, "%+0.8le ", v[i * (uint64_t)R + j]);
                        o.append(buf, (size_t)k);
                    }
                    o += '\n';
                }
            };
            host_run(P, fmt);
            for (int q = 0; q < P && ok; ++q)
                ok = fwrite(out[q].data(), 1, out[q].size(), f) == out[q].size();
        }
        if (!ok) {
            fclose(f);
            fail(CTC_E_IO, "write to %s failed", path);
        }
        if (fclose(f) != 0) fail(CTC_E_IO, "closing %s failed", path);
    });
}

// Exact binary checkpoint of a model (factors in FP64, bit for bit):
//   "CTCM" | u32 version 1 | u32 nmodes | u32 rank | u64 dims[nmodes] |
//   f64 rows of mode 0 (row-major) | ... | f64 rows of the last mode
static const char kModelMagic[4] = {'C', 'T', 'C', 'M'};

extern "C" int ctc_model_save(const ctc_model *m, const char *path)
{
    return guarded([&] {
        if (!m || !path || m->nmodes < 1) fail(CTC_E_ARG, "bad argument");
        FILE *f = fopen(path, "wb");
        if (!f) fail(CTC_E_IO, "cannot open %s for writing", path);
        const uint32_t hdr[3] = {1u, (uint32_t)m->nmodes, (uint32_t)m->rank};
        bool ok = fwrite(kModelMagic, 1, 4, f) == 4 && fwrite(hdr, 4, 3, f) == 3 &&
                  fwrite(m->dims, 8, (size_t)m->nmodes, f) == (size_t)m->nmodes;
        for (int k = 0; ok && k < m->nmodes; ++k)
            ok = fwrite(m->U[k].data(), 8, m->U[k].size(), f) == m->U[k].size();
        if (fclose(f) != 0) ok = false;
        if (!ok) fail(CTC_E_IO, "write to %s failed", path);
    });
}

extern "C" int ctc_model_load(const char *path, ctc_model **out)
{
    return guarded([&] {
        if (!path || !out) fail(CTC_E_ARG, "null argument");
        FILE *f = fopen(path, "rb");
        if (!f) fail(CTC_E_IO, "cannot open %s", path);
        std::unique_ptr<FILE, int (*)(FILE *)> guard(f, fclose);
        char magic[4];
        uint32_t hdr[3];
        if (fread(magic, 1, 4, f) != 4 || memcmp(magic, kModelMagic, 4) != 0 || fread(hdr, 4, 3, f) != 3)
            fail(CTC_E_IO, "%s is not a model checkpoint", path);
        if (hdr[0] != 1u) fail(CTC_E_IO, "%s: checkpoint version %u", path, hdr[0]);
        if (hdr[1] < 1 || hdr[1] > 4 || hdr[2] < 1 || hdr[2] > 4096) fail(CTC_E_IO, "%s: bad shape", path);
        auto m = std::make_unique<ctc_model>();
        m->nmodes = (int)hdr[1];
        m->rank = (int)hdr[2];
        if (fread(m->dims, 8, (size_t)m->nmodes, f) != (size_t)m->nmodes) fail(CTC_E_IO, "%s: truncated", path);
        for (int k = 0; k < m->nmodes; ++k) {
            if (m->dims[k] == 0 || m->dims[k] > ((uint64_t)1 << 40)) fail(CTC_E_IO, "%s: bad dimension", path);
            m->U[k].resize(m->dims[k] * (uint64_t)m->rank);
            if (fread(m->U[k].data(), 8, m->U[k].size(), f) != m->U[k].size())
                fail(CTC_E_IO, "%s: truncated", path);
        }
        *out = m.release();
    });
}

extern "C" int ctc_model_copy(const ctc_model *src, ctc_model *dst)
{
    return guarded([&] {
        if (!src || !dst) fail(CTC_E_ARG, "null model");
        *dst = *src;
    });
}

extern "C" int ctc_model_info(const ctc_model *m, int *nmodes, uint64_t *dims, int *rank)
{
    return guarded([&] {
        if (!m) fail(CTC_E_ARG, "null model");
        if (nmodes) *nmodes = m->nmodes;
        if (rank) *rank = m->rank;
        if (dims)
            for (int q = 0; q < m->nmodes; ++q) dims[q] = m->dims[q];
    });
}

extern "C" int ctc_model_free(ctc_model *m)
{
    delete m;
    return CTC_OK;
}
