// Record file format of the reference (README.md:41-61):
//   "R H" header, R read lines of 5 equal-length fields
//   (bases, base/ins/del/gcp quality), H haplotype lines.
// Output: "R H" then R lines of H "%.5f" scores separated by single spaces.
//
// Both directions run on several host threads: the reference's parser and
// writer are single threads (file_parser_worker.cu:88-153,
// output_writer_worker.cu:84-135) and bound a file-to-file run once the GPU
// part is fast.
#pragma once

#include <cstdint>
#include <cstdio>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/pairhmm_b200.h"

namespace phmm {

// Allocator whose value-less construct leaves elements uninitialised, so that
// resize() ahead of a parallel fill does not write every byte twice.
template <class T>
struct NoInitAllocator : std::allocator<T> {
    using value_type = T;
    NoInitAllocator() noexcept = default;
    template <class U>
    NoInitAllocator(const NoInitAllocator<U>&) noexcept {}
    template <class U>
    struct rebind {
        using other = NoInitAllocator<U>;
    };
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using HostVector = std::vector<T, NoInitAllocator<T>>;

// Threads used by the parser and the formatter: set_host_threads(n) with n > 0,
// else the PAIRHMM_HOST_THREADS environment variable, else the hardware
// threads; at most 64.
int host_threads();
void set_host_threads(int n);

// Structure-of-arrays batch on the host (the reference's BatchOfSequenceGroups,
// common.cuh:109-201).  Reads and haplotypes are padded like the reference
// parser pads them (4 - len%4 bytes of 'N', quality 'N'-33;
// file_parser_worker.cu:81-86), so offsets stay 4-byte aligned.
struct HostBatch {
    HostVector<int32_t> reads_per_record, haps_per_record;
    HostVector<uint8_t> read_bases, base_quals, ins_quals, del_quals, gcp_quals;
    HostVector<int64_t> read_offsets;
    HostVector<int32_t> read_lengths;
    HostVector<uint8_t> hap_bases;
    HostVector<int64_t> hap_offsets;
    HostVector<int32_t> hap_lengths;
    int64_t pairs = 0;

    void clear();
    int64_t num_records() const { return (int64_t)reads_per_record.size(); }
    pairhmm_batch_t view() const;
};

// Streaming parser (file_parser_worker.cu:50-153).  next() appends whole
// records until the batch holds at least min_pairs pairs or the input ends.
// A regular file is mapped, other files are read whole; a text buffer given
// to the second constructor is used in place and must outlive the reader.
//
// next() indexes the newlines ahead of it on all host threads, walks the
// record headers over that index on one thread, then checks the read and
// haplotype lines and copies and decodes them on all host threads.  Errors
// name the 1-based line; when several lines are malformed the first is named.
class RecordReader {
public:
    explicit RecordReader(const std::string& path);
    RecordReader(const char* text, size_t size);
    ~RecordReader();
    RecordReader(const RecordReader&) = delete;
    RecordReader& operator=(const RecordReader&) = delete;
    bool ok() const { return !open_failed_; }
    // returns false on a malformed record (message in error()); true otherwise
    bool next(HostBatch& out, int64_t min_pairs, bool& eof);
    const std::string& error() const { return err_; }

private:
    void index_more(int64_t bytes);
    bool have_line(size_t k, int64_t& chunk);
    const char* data_ = nullptr;
    int64_t size_ = 0;
    int64_t pos_ = 0;      // first byte not consumed
    int64_t line_no_ = 0;  // lines consumed
    void* map_ = nullptr;
    size_t map_size_ = 0;
    std::vector<char> owned_;
    bool open_failed_ = false;
    std::string err_;
    HostVector<int64_t> ends_;  // line ends from pos_ on, as far as indexed
    size_t consumed_ = 0;       // leading entries of ends_ consumed by the last next()
    int64_t indexed_to_ = 0;    // newlines are indexed up to here
};

// Parses a whole text buffer.
bool parse_records(const char* text, size_t size, HostBatch& out, std::string& err);
inline bool parse_records(const std::string& text, HostBatch& out, std::string& err) {
    return parse_records(text.data(), text.size(), out, err);
}

// Writes x as printf("%.5f", x) does with the C library's round-to-nearest:
// the exact binary value rounded to 5 decimals, ties to even, "-" for every
// negative value (also "-0.00000"), "inf"/"nan" with their sign.  Needs 64
// bytes of room at p; returns the end of the text.
char* put_fixed5(char* p, float x);

// The output lines of a batch (output_writer_worker.cu:107-135), formatted on
// several threads into consecutive parts whose concatenation is the text.
void format_scores_parts(const HostBatch& b, const float* scores, std::vector<std::string>& parts);
// The same text appended to out.
void format_scores(const HostBatch& b, const float* scores, std::string& out);

}  // namespace phmm
