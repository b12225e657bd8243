// Record file format of the reference (README.md:41-61):
//   "R H" header, R read lines of 5 equal-length fields
//   (bases, base/ins/del/gcp quality), H haplotype lines.
// Output: "R H" then R lines of H "%.5f" scores separated by single spaces.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/pairhmm_b200.h"

namespace phmm {

// Structure-of-arrays batch on the host (the reference's BatchOfSequenceGroups,
// common.cuh:109-201).  Reads and haplotypes are padded like the reference
// parser pads them (4 - len%4 bytes of 'N', quality 'N'-33;
// file_parser_worker.cu:81-86), so offsets stay 4-byte aligned.
struct HostBatch {
    std::vector<int32_t> reads_per_record, haps_per_record;
    std::vector<uint8_t> read_bases, base_quals, ins_quals, del_quals, gcp_quals;
    std::vector<int64_t> read_offsets;
    std::vector<int32_t> read_lengths;
    std::vector<uint8_t> hap_bases;
    std::vector<int64_t> hap_offsets;
    std::vector<int32_t> hap_lengths;
    int64_t pairs = 0;

    void clear();
    int64_t num_records() const { return (int64_t)reads_per_record.size(); }
    pairhmm_batch_t view() const;
};

// Streaming parser (file_parser_worker.cu:50-153).  next() appends whole
// records until the batch holds at least min_pairs pairs or the file ends.
class RecordReader {
public:
    explicit RecordReader(const std::string& path);
    ~RecordReader();
    bool ok() const { return f_ != nullptr; }
    // returns false on a malformed record (message in error()); true otherwise
    bool next(HostBatch& out, int64_t min_pairs, bool& eof);
    const std::string& error() const { return err_; }

private:
    bool getline(std::string& line);
    FILE* f_ = nullptr;
    std::vector<char> buf_;
    size_t pos_ = 0, len_ = 0;
    bool eof_ = false;
    int64_t line_no_ = 0;
    std::string err_;
};

// Parses a whole text buffer (tests, small inputs).
bool parse_records(const std::string& text, HostBatch& out, std::string& err);

// Appends the output lines for a batch (output_writer_worker.cu:107-135).
void format_scores(const HostBatch& b, const float* scores, std::string& out);

}  // namespace phmm
