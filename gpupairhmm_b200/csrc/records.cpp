#include "records.hpp"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <mutex>
#include <thread>

namespace phmm {

namespace {

// file_parser_worker.cu:81-86: always 1..4 bytes of padding
inline int64_t pad_len(int64_t n) { return 4 - (n % 4); }
constexpr uint8_t kPadBase = 'N';
constexpr uint8_t kPadQual = 'N' - 33;

std::atomic<int> g_host_threads{0};

// Runs f(task) for task in [0, ntasks) on up to `threads` threads (the caller
// is one of them); the first exception thrown by a task is rethrown here.
template <class F>
void run_tasks(int64_t ntasks, int threads, F&& f) {
    threads = (int)std::min<int64_t>(threads, ntasks);
    if (threads <= 1) {
        for (int64_t t = 0; t < ntasks; ++t) f(t);
        return;
    }
    std::atomic<int64_t> next{0};
    std::exception_ptr failure;
    std::mutex m;
    auto work = [&] {
        try {
            for (int64_t t; (t = next.fetch_add(1)) < ntasks;) f(t);
        } catch (...) {
            std::lock_guard<std::mutex> lk(m);
            if (!failure) failure = std::current_exception();
            next.store(ntasks);
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(threads - 1);
    for (int i = 1; i < threads; ++i) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (failure) std::rethrow_exception(failure);
}

// Cuts [0, n) into about `parts` ranges of equal weight; weight_before(i) is
// the total weight of items [0, i) (non-decreasing).
template <class W>
std::vector<int64_t> balanced_cuts(int64_t n, int64_t parts, W&& weight_before) {
    std::vector<int64_t> cuts{0};
    const int64_t total = weight_before(n);
    for (int64_t k = 1; k < parts; ++k) {
        const int64_t target = total / parts * k;
        int64_t lo = cuts.back(), hi = n;  // first i with weight_before(i) >= target
        while (lo < hi) {
            const int64_t mid = lo + (hi - lo) / 2;
            if (weight_before(mid) < target) lo = mid + 1;
            else hi = mid;
        }
        if (lo > cuts.back() && lo < n) cuts.push_back(lo);
    }
    cuts.push_back(n);
    return cuts;
}

// Threads worth starting for `bytes` of work (about 1 MB each at least).
int threads_for(int64_t bytes) {
    return (int)std::max<int64_t>(1, std::min<int64_t>(host_threads(), bytes >> 20));
}

bool parse_header(const char* s, size_t n, int64_t& R, int64_t& H) {
    const std::string line(s, n);
    const size_t sp = line.find(' ');
    if (sp == std::string::npos || sp == 0) return false;
    char* end = nullptr;
    errno = 0;
    R = std::strtoll(line.c_str(), &end, 10);
    if (end != line.c_str() + sp || errno) return false;
    const char* p = line.c_str() + sp;
    H = std::strtoll(p, &end, 10);
    if (end == p || errno) return false;
    return R >= 0 && H >= 0 && R < (int64_t(1) << 31) && H < (int64_t(1) << 31);
}

struct Planned {
    int64_t first_line;    // the header's line, counted from the reader's position
    int32_t R, H;
    int64_t read0, hap0;   // the record's first read and haplotype in this call
};

}  // namespace

int host_threads() {
    int n = g_host_threads.load();
    if (n <= 0) {
        const char* e = std::getenv("PAIRHMM_HOST_THREADS");
        n = e ? std::atoi(e) : 0;
        if (n <= 0) n = (int)std::thread::hardware_concurrency();
    }
    return std::max(1, std::min(n, 64));
}

void set_host_threads(int n) { g_host_threads.store(n > 0 ? n : 0); }

void HostBatch::clear() {
    reads_per_record.clear();
    haps_per_record.clear();
    read_bases.clear();
    base_quals.clear();
    ins_quals.clear();
    del_quals.clear();
    gcp_quals.clear();
    read_offsets.clear();
    read_lengths.clear();
    hap_bases.clear();
    hap_offsets.clear();
    hap_lengths.clear();
    pairs = 0;
}

pairhmm_batch_t HostBatch::view() const {
    pairhmm_batch_t v{};
    v.num_records = num_records();
    v.reads_per_record = reads_per_record.data();
    v.haps_per_record = haps_per_record.data();
    v.read_bases = read_bases.data();
    v.base_quals = base_quals.data();
    v.ins_quals = ins_quals.data();
    v.del_quals = del_quals.data();
    v.gcp_quals = gcp_quals.data();
    v.read_offsets = read_offsets.data();
    v.read_lengths = read_lengths.data();
    v.hap_bases = hap_bases.data();
    v.hap_offsets = hap_offsets.data();
    v.hap_lengths = hap_lengths.data();
    return v;
}

RecordReader::RecordReader(const std::string& path) {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) {
        open_failed_ = true;
        size_ = -1;
        err_ = "could not open file " + path;
        return;
    }
    struct stat st{};
    if (::fstat(fd, &st) == 0 && S_ISREG(st.st_mode)) {
        size_ = (int64_t)st.st_size;
        if (size_ > 0) {
            void* p = ::mmap(nullptr, (size_t)size_, PROT_READ, MAP_PRIVATE, fd, 0);
            if (p != MAP_FAILED) {
                ::madvise(p, (size_t)size_, MADV_SEQUENTIAL);
                ::madvise(p, (size_t)size_, MADV_WILLNEED);
                map_ = p;
                map_size_ = (size_t)size_;
                data_ = static_cast<const char*>(p);
            }
        }
    }
    if (!map_) {  // a pipe, a device, or a file that could not be mapped: read it whole
        size_ = 0;
        owned_.resize(size_t(1) << 22);
        for (;;) {
            if ((size_t)size_ == owned_.size()) owned_.resize(owned_.size() * 2);
            const ssize_t got = ::read(fd, owned_.data() + size_, owned_.size() - (size_t)size_);
            if (got < 0 && errno == EINTR) continue;
            if (got < 0) {
                open_failed_ = true;
                err_ = "could not read file " + path;
                break;
            }
            if (got == 0) break;
            size_ += got;
        }
        data_ = owned_.data();
        if (open_failed_) size_ = -1;
    }
    ::close(fd);
}

RecordReader::RecordReader(const char* text, size_t size) : data_(text), size_((int64_t)size) {}

RecordReader::~RecordReader() {
    if (map_) ::munmap(map_, map_size_);
}

void RecordReader::index_more(int64_t bytes) {
    // newline positions of [indexed_to_, indexed_to_ + bytes), found by all
    // host threads over equal slices and appended in order
    const int64_t a = indexed_to_, b = std::min(size_, a + bytes);
    const int threads = threads_for(b - a);
    std::vector<HostVector<int64_t>> found((size_t)threads);
    run_tasks(threads, threads, [&](int64_t t) {
        const int64_t lo = a + (b - a) * t / threads, hi = a + (b - a) * (t + 1) / threads;
        HostVector<int64_t>& v = found[t];
        v.reserve((size_t)((hi - lo) / 256 + 16));
        for (int64_t x = lo; x < hi;) {
            const void* nl = std::memchr(data_ + x, '\n', (size_t)(hi - x));
            if (!nl) break;
            const int64_t e = static_cast<const char*>(nl) - data_;
            v.push_back(e);
            x = e + 1;
        }
    });
    size_t n = ends_.size();
    for (const auto& v : found) n += v.size();
    ends_.reserve(n + 1);
    for (const auto& v : found) ends_.insert(ends_.end(), v.begin(), v.end());
    indexed_to_ = b;
    // a last line without a newline ends at the end of the input
    if (b == size_ && size_ > 0 && data_[size_ - 1] != '\n' &&
        (ends_.empty() ? pos_ < size_ : ends_.back() + 1 < size_))
        ends_.push_back(size_);
}

bool RecordReader::have_line(size_t k, int64_t& chunk) {
    while (ends_.size() <= k && indexed_to_ < size_) {
        index_more(chunk);
        chunk = std::min<int64_t>(chunk * 2, int64_t(1) << 30);
    }
    return ends_.size() > k;
}

bool RecordReader::next(HostBatch& out, int64_t min_pairs, bool& eof) {
    eof = false;
    if (open_failed_) return false;
    // Lines already consumed leave the index; ends_[k] is then the end of the
    // k-th line from pos_ (a newline's position, or size_ for a last line
    // without one), and line k starts at pos_ (k = 0) or ends_[k-1] + 1.
    ends_.erase(ends_.begin(), ends_.begin() + (ptrdiff_t)consumed_);
    consumed_ = 0;
    auto start = [&](size_t k) { return k == 0 ? pos_ : ends_[k - 1] + 1; };
    int64_t chunk = int64_t(64) << 20;

    // Step 1 (one thread): the record structure from the line index.  Only
    // header lines are read.
    std::vector<Planned> recs;
    size_t k = 0;
    int64_t pairs = out.pairs, nrec = out.num_records(), nreads = 0, nhaps = 0;
    std::string err;
    int64_t err_line = std::numeric_limits<int64_t>::max();
    while (pairs < min_pairs || nrec == 0) {
        while (have_line(k, chunk) && start(k) == ends_[k]) ++k;  // blank separator lines
        if (!have_line(k, chunk)) {
            eof = true;
            break;
        }
        int64_t R = 0, H = 0;
        if (!parse_header(data_ + start(k), (size_t)(ends_[k] - start(k)), R, H)) {
            err = "malformed record header";
            err_line = line_no_ + (int64_t)k + 1;
            break;
        }
        if (!have_line(k + (size_t)(R + H), chunk)) {
            const int64_t lines = (int64_t)ends_.size() - (int64_t)k - 1;  // lines after the header
            err = lines < R ? "file ends inside a record's reads" : "file ends inside a record's haplotypes";
            err_line = line_no_ + (int64_t)ends_.size();  // the last line of the input
            break;
        }
        recs.push_back({(int64_t)k, (int32_t)R, (int32_t)H, nreads, nhaps});
        nreads += R;
        nhaps += H;
        pairs += R * H;
        ++nrec;
        k += 1 + (size_t)(R + H);
    }

    // Step 2 (all threads): line checks and lengths of every read and haplotype.
    const size_t read0 = out.read_lengths.size(), hap0 = out.hap_lengths.size();
    const int64_t rb0 = (int64_t)out.read_bases.size(), hb0 = (int64_t)out.hap_bases.size();
    auto undo = [&] {  // leaves `out` as it was before the call
        out.read_lengths.resize(read0);
        out.read_offsets.resize(read0);
        out.hap_lengths.resize(hap0);
        out.hap_offsets.resize(hap0);
        for (auto* v : {&out.read_bases, &out.base_quals, &out.ins_quals, &out.del_quals, &out.gcp_quals})
            v->resize((size_t)rb0);
        out.hap_bases.resize((size_t)hb0);
    };
    out.read_lengths.resize(read0 + (size_t)nreads);
    out.read_offsets.resize(read0 + (size_t)nreads);
    out.hap_lengths.resize(hap0 + (size_t)nhaps);
    out.hap_offsets.resize(hap0 + (size_t)nhaps);
    const int64_t nr = (int64_t)recs.size();
    const int64_t text_bytes = nr ? ends_[recs.back().first_line + recs.back().R + recs.back().H] - pos_ : 0;
    int threads = threads_for(text_bytes);
    std::vector<int64_t> cuts = balanced_cuts(nr, (int64_t)threads * 4, [&](int64_t g) {
        return g < nr ? start((size_t)recs[g].first_line) - pos_ : text_bytes;
    });
    std::atomic<int64_t> bad_line{std::numeric_limits<int64_t>::max()};
    std::atomic<int> bad_kind{0};
    std::mutex bad_m;
    auto report = [&](int64_t line, int kind) {
        std::lock_guard<std::mutex> lk(bad_m);
        if (line < bad_line.load()) {
            bad_line.store(line);
            bad_kind.store(kind);
        }
    };
    int32_t* rlen = out.read_lengths.data() + read0;
    int32_t* hlen = out.hap_lengths.data() + hap0;
    run_tasks((int64_t)cuts.size() - 1, threads, [&](int64_t t) {
        for (int64_t g = cuts[t]; g < cuts[t + 1]; ++g) {
            const Planned& p = recs[g];
            size_t line = (size_t)p.first_line + 1;
            for (int32_t r = 0; r < p.R; ++r, ++line) {
                const int64_t s = start(line), n = ends_[line] - s;
                const void* sp = std::memchr(data_ + s, ' ', (size_t)n);
                const int64_t L = sp ? static_cast<const char*>(sp) - (data_ + s) : 0;
                if (L == 0) report(line_no_ + (int64_t)line + 1, 1);
                else if (n < 5 * L + 4) report(line_no_ + (int64_t)line + 1, 2);
                rlen[p.read0 + r] = (int32_t)L;
            }
            for (int32_t h = 0; h < p.H; ++h, ++line) {
                const int64_t n = ends_[line] - start(line);
                if (n == 0) report(line_no_ + (int64_t)line + 1, 3);
                hlen[p.hap0 + h] = (int32_t)n;
            }
        }
    });
    if (bad_line.load() < err_line) {  // every planned record comes before the walk's stop
        static const char* kMsg[] = {"", "read line without 5 space-separated fields",
                                     "read line shorter than 5 fields of the read length", "empty haplotype line"};
        err = kMsg[bad_kind.load()];
        err_line = bad_line.load();
    }
    if (!err.empty()) {
        err_ = err + " (line " + std::to_string(err_line) + ")";
        undo();
        return false;
    }

    // Step 3: offsets (prefix sums), then all threads copy and decode.
    int64_t read_bytes = rb0, hap_bytes = hb0;
    int64_t* roff = out.read_offsets.data() + read0;
    int64_t* hoff = out.hap_offsets.data() + hap0;
    for (int64_t i = 0; i < nreads; ++i) {
        roff[i] = read_bytes;
        read_bytes += rlen[i] + pad_len(rlen[i]);
    }
    for (int64_t j = 0; j < nhaps; ++j) {
        hoff[j] = hap_bytes;
        hap_bytes += hlen[j] + pad_len(hlen[j]);
    }
    try {
        for (auto* v : {&out.read_bases, &out.base_quals, &out.ins_quals, &out.del_quals, &out.gcp_quals})
            v->resize((size_t)read_bytes);
        out.hap_bases.resize((size_t)hap_bytes);
    } catch (...) {
        undo();
        throw;
    }
    uint8_t* qv[4] = {out.base_quals.data(), out.ins_quals.data(), out.del_quals.data(), out.gcp_quals.data()};
    uint8_t* rbases = out.read_bases.data();
    uint8_t* hbases = out.hap_bases.data();
    threads = threads_for((read_bytes - rb0) * 5 + (hap_bytes - hb0));
    cuts = balanced_cuts(nr, (int64_t)threads * 4, [&](int64_t g) {
        return g < nr ? start((size_t)recs[g].first_line) - pos_ : text_bytes;
    });
    run_tasks((int64_t)cuts.size() - 1, threads, [&](int64_t t) {
        for (int64_t g = cuts[t]; g < cuts[t + 1]; ++g) {
            const Planned& p = recs[g];
            size_t line = (size_t)p.first_line + 1;
            for (int32_t r = 0; r < p.R; ++r, ++line) {
                const int64_t i = p.read0 + r, L = rlen[i], o = roff[i], pad = pad_len(L);
                const uint8_t* s = reinterpret_cast<const uint8_t*>(data_ + start(line));
                std::memcpy(rbases + o, s, (size_t)L);
                std::memset(rbases + o + L, kPadBase, (size_t)pad);
                for (int q = 0; q < 4; ++q) {
                    const uint8_t* f = s + (q + 1) * (L + 1);
                    uint8_t* d = qv[q] + o;
                    for (int64_t x = 0; x < L; ++x) d[x] = (uint8_t)(f[x] - 33);  // file_parser_worker.cu:95
                    std::memset(d + L, kPadQual, (size_t)pad);
                }
            }
            for (int32_t h = 0; h < p.H; ++h, ++line) {
                const int64_t j = p.hap0 + h, n = hlen[j], o = hoff[j];
                std::memcpy(hbases + o, data_ + start(line), (size_t)n);
                std::memset(hbases + o + n, kPadBase, (size_t)pad_len(n));
            }
        }
    });
    for (const Planned& p : recs) {
        out.reads_per_record.push_back(p.R);
        out.haps_per_record.push_back(p.H);
    }
    out.pairs = pairs;
    // consume through the last planned record (and blank lines before the end)
    const size_t take = std::min(k, ends_.size());
    if (take > 0) {
        pos_ = std::min(size_, ends_[take - 1] + 1);
        line_no_ += (int64_t)take;
        consumed_ = take;
    }
    return true;
}

bool parse_records(const char* text, size_t size, HostBatch& out, std::string& err) {
    RecordReader r(text, size);
    bool eof = false;
    if (!r.next(out, std::numeric_limits<int64_t>::max(), eof)) {
        err = r.error();
        return false;
    }
    return true;
}

namespace {

inline char* put_uint(char* p, uint64_t v) {
    char tmp[20];
    int n = 0;
    do {
        tmp[n++] = char('0' + v % 10);
        v /= 10;
    } while (v);
    while (n) *p++ = tmp[--n];
    return p;
}

}  // namespace

char* put_fixed5(char* p, float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t ebits = (u >> 23) & 0xffu, frac = u & 0x7fffffu;
    const bool neg = (u >> 31) != 0;
    if (ebits == 0xffu) {
        if (neg) *p++ = '-';
        std::memcpy(p, frac ? "nan" : "inf", 3);
        return p + 3;
    }
    // x = m * 2^e exactly; N = x * 10^5 rounded to the nearest integer, ties to even
    const uint64_t m = ebits ? (frac | 0x800000u) : frac;
    const int e = ebits ? (int)ebits - 150 : -149;
    if (e > 0) return p + std::snprintf(p, 64, "%.5f", (double)x);  // |x| >= 2^24: not a log10 score
    const uint64_t P = m * 100000u;  // < 2^41
    const int k = -e;
    uint64_t N;
    if (k == 0) {
        N = P;
    } else if (k >= 63) {
        N = 0;  // x * 10^5 < 2^-22
    } else {
        N = P >> k;
        const uint64_t r = P & ((uint64_t(1) << k) - 1), half = uint64_t(1) << (k - 1);
        if (r > half || (r == half && (N & 1))) ++N;
    }
    if (neg) *p++ = '-';
    p = put_uint(p, N / 100000u);
    *p++ = '.';
    uint32_t f = (uint32_t)(N % 100000u);
    for (int d = 4; d >= 0; --d) {
        p[d] = char('0' + f % 10);
        f /= 10;
    }
    return p + 5;
}

void format_scores_parts(const HostBatch& b, const float* scores, std::vector<std::string>& parts) {
    const int64_t ng = b.num_records();
    // pairs before record g, for the cut and for each part's first score
    std::vector<int64_t> pair_before((size_t)ng + 1, 0);
    for (int64_t g = 0; g < ng; ++g)
        pair_before[g + 1] = pair_before[g] + (int64_t)b.reads_per_record[g] * b.haps_per_record[g];
    const int threads = threads_for(pair_before[ng] * 10);
    const std::vector<int64_t> cuts = balanced_cuts(ng, (int64_t)threads * 4, [&](int64_t g) {
        return pair_before[g] + g;  // + g: a record's header line also costs
    });
    const int64_t ntasks = (int64_t)cuts.size() - 1;
    parts.assign((size_t)std::max<int64_t>(ntasks, 0), std::string());
    run_tasks(ntasks, threads, [&](int64_t t) {
        std::string& s = parts[t];
        size_t used = 0;
        auto room = [&](size_t need) {
            if (used + need > s.size()) s.resize(std::max(s.size() * 2, used + need));
        };
        room((size_t)(pair_before[cuts[t + 1]] - pair_before[cuts[t]]) * 11 + 64);
        int64_t k = pair_before[cuts[t]];
        for (int64_t g = cuts[t]; g < cuts[t + 1]; ++g) {
            const int R = b.reads_per_record[g], H = b.haps_per_record[g];
            room(48);
            char* p = &s[used];
            char* q = put_uint(p, (uint64_t)R);
            *q++ = ' ';
            q = put_uint(q, (uint64_t)H);
            *q++ = '\n';
            used += q - p;
            for (int r = 0; r < R; ++r) {
                room((size_t)H * 65 + 1);
                p = &s[used];
                q = p;
                for (int h = 0; h < H; ++h) {
                    if (h > 0) *q++ = ' ';
                    q = put_fixed5(q, scores[k++]);
                }
                *q++ = '\n';
                used += q - p;
            }
        }
        s.resize(used);
    });
}

void format_scores(const HostBatch& b, const float* scores, std::string& out) {
    std::vector<std::string> parts;
    format_scores_parts(b, scores, parts);
    size_t n = out.size();
    for (const auto& s : parts) n += s.size();
    out.reserve(n);
    for (const auto& s : parts) out += s;
}

}  // namespace phmm
