#include "records.hpp"

#include <cerrno>
#include <cstdlib>
#include <cstring>

namespace phmm {

namespace {

// file_parser_worker.cu:81-86: always 1..4 bytes of padding
inline int pad_len(int n) { return 4 - (n % 4); }
constexpr uint8_t kPadBase = 'N';
constexpr uint8_t kPadQual = 'N' - 33;

bool parse_header(const std::string& line, int64_t& R, int64_t& H) {
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

template <class NextLine>
bool parse_record(NextLine&& next_line, int64_t R, int64_t H, HostBatch& b, std::string& err) {
    std::string line;
    for (int64_t r = 0; r < R; ++r) {
        if (!next_line(line)) { err = "file ends inside a record's reads"; return false; }
        const size_t L = line.find(' ');
        if (L == std::string::npos || L == 0) { err = "read line without 5 space-separated fields"; return false; }
        if (line.size() < 5 * L + 4) { err = "read line shorter than 5 fields of the read length"; return false; }
        const int pad = pad_len((int)L);
        const int64_t start = (int64_t)b.read_bases.size();
        b.read_offsets.push_back(start);
        b.read_lengths.push_back((int32_t)L);
        const uint8_t* s = reinterpret_cast<const uint8_t*>(line.data());
        b.read_bases.insert(b.read_bases.end(), s, s + L);
        b.read_bases.insert(b.read_bases.end(), pad, kPadBase);
        std::vector<uint8_t>* qv[4] = {&b.base_quals, &b.ins_quals, &b.del_quals, &b.gcp_quals};
        for (int k = 0; k < 4; ++k) {
            const uint8_t* f = s + (k + 1) * (L + 1);
            std::vector<uint8_t>& q = *qv[k];
            const size_t o = q.size();
            q.resize(o + L + pad);
            for (size_t i = 0; i < L; ++i) q[o + i] = (uint8_t)(f[i] - 33);  // file_parser_worker.cu:95
            std::memset(&q[o + L], kPadQual, pad);
        }
    }
    for (int64_t h = 0; h < H; ++h) {
        if (!next_line(line)) { err = "file ends inside a record's haplotypes"; return false; }
        const size_t n = line.size();
        if (n == 0) { err = "empty haplotype line"; return false; }
        b.hap_offsets.push_back((int64_t)b.hap_bases.size());
        b.hap_lengths.push_back((int32_t)n);
        const uint8_t* s = reinterpret_cast<const uint8_t*>(line.data());
        b.hap_bases.insert(b.hap_bases.end(), s, s + n);
        b.hap_bases.insert(b.hap_bases.end(), pad_len((int)n), kPadBase);
    }
    b.reads_per_record.push_back((int32_t)R);
    b.haps_per_record.push_back((int32_t)H);
    b.pairs += R * H;
    return true;
}

}  // namespace

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

RecordReader::RecordReader(const std::string& path) : buf_(size_t(1) << 22) {
    f_ = std::fopen(path.c_str(), "rb");
    if (!f_) err_ = "could not open file " + path;
}

RecordReader::~RecordReader() {
    if (f_) std::fclose(f_);
}

bool RecordReader::getline(std::string& line) {
    line.clear();
    for (;;) {
        if (pos_ == len_) {
            if (eof_) return !line.empty();
            len_ = std::fread(buf_.data(), 1, buf_.size(), f_);
            pos_ = 0;
            if (len_ == 0) {
                eof_ = true;
                return !line.empty();
            }
        }
        const char* start = buf_.data() + pos_;
        const void* nl = std::memchr(start, '\n', len_ - pos_);
        if (nl) {
            const size_t n = static_cast<const char*>(nl) - start;
            line.append(start, n);
            pos_ += n + 1;
            ++line_no_;
            return true;
        }
        line.append(start, len_ - pos_);
        pos_ = len_;
    }
}

bool RecordReader::next(HostBatch& out, int64_t min_pairs, bool& eof) {
    eof = false;
    std::string header;
    while (out.pairs < min_pairs || out.num_records() == 0) {
        if (!getline(header)) {
            eof = true;
            return true;
        }
        if (header.empty()) continue;  // blank separator lines are skipped
        int64_t R = 0, H = 0;
        if (!parse_header(header, R, H)) {
            err_ = "malformed record header at line " + std::to_string(line_no_);
            return false;
        }
        auto nl = [this](std::string& l) { return getline(l); };
        if (!parse_record(nl, R, H, out, err_)) {
            err_ += " (line " + std::to_string(line_no_) + ")";
            return false;
        }
    }
    return true;
}

bool parse_records(const std::string& text, HostBatch& out, std::string& err) {
    size_t pos = 0;
    auto next_line = [&](std::string& l) {
        if (pos >= text.size()) return false;
        const size_t nl = text.find('\n', pos);
        const size_t end = nl == std::string::npos ? text.size() : nl;
        l.assign(text, pos, end - pos);
        pos = nl == std::string::npos ? text.size() : nl + 1;
        return true;
    };
    std::string header;
    while (next_line(header)) {
        if (header.empty()) continue;
        int64_t R = 0, H = 0;
        if (!parse_header(header, R, H)) {
            err = "malformed record header";
            return false;
        }
        if (!parse_record(next_line, R, H, out, err)) return false;
    }
    return true;
}

void format_scores(const HostBatch& b, const float* scores, std::string& out) {
    char tmp[64];
    int64_t k = 0;
    for (size_t g = 0; g < b.reads_per_record.size(); ++g) {
        const int R = b.reads_per_record[g], H = b.haps_per_record[g];
        int n = std::snprintf(tmp, sizeof(tmp), "%d %d\n", R, H);
        out.append(tmp, n);
        for (int r = 0; r < R; ++r) {
            for (int h = 0; h < H; ++h) {
                if (h > 0) out.push_back(' ');
                n = std::snprintf(tmp, sizeof(tmp), "%.5f", scores[k++]);
                out.append(tmp, n);
            }
            out.push_back('\n');
        }
    }
}

}  // namespace phmm
