// FASTA/FASTQ (plain or gzip) -> sufkit logical text, for sufgpu_encode_fasta.
//
// Follows GenomeReference::FromFasta (src/genome_reference.cpp:222-268) as fed
// by kseq (third_party/kseq/kseq.h): a record starts at '>' or '@'; its name
// runs to the first whitespace and the rest of the header line is the
// description; sequence lines are concatenated (empty lines skipped, a final
// '\r' dropped once the sequence holds more than one byte) until a line starts
// with '>', '@' or '+'; '+' begins a FASTQ quality block of the same length.
// Bytes are normalized by the encoding table of src/genome_reference.cpp:30-46
// (A/C/G/T any case -> 2..5, anything else -> 6) and a 1 follows every record
// (src/genome_reference.cpp:147-149).  Records must have unique non-empty
// names and non-empty sequences (src/genome_reference.cpp:88-122).

#include <zlib.h>

#include <cctype>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/sufgpu/sufgpu.h"

namespace {

class Reader {
 public:
  explicit Reader(gzFile f) : f_(f), buf_(1 << 20) {}
  // Next byte or -1 at end of input, -3 on a stream error.
  int get() {
    if (pos_ == len_) {
      if (eof_) return -1;
      const int got = gzread(f_, buf_.data(), static_cast<unsigned>(buf_.size()));
      if (got < 0) return -3;
      if (got == 0) {
        eof_ = true;
        return -1;
      }
      len_ = static_cast<size_t>(got);
      pos_ = 0;
    }
    return buf_[pos_++];
  }

 private:
  gzFile f_;
  std::vector<unsigned char> buf_;
  size_t pos_ = 0, len_ = 0;
  bool eof_ = false;
};

struct Record {
  std::string name;
  std::string seq;
};

// Reads the rest of a line (the '\n' is consumed, not stored).
int read_line(Reader& r, std::string& into) {
  int c;
  while ((c = r.get()) >= 0 && c != '\n') into.push_back(static_cast<char>(c));
  return c == -3 ? -3 : 0;
}

uint8_t encode_base(unsigned char c) {
  switch (c) {
    case 'A': case 'a': return 2;
    case 'C': case 'c': return 3;
    case 'G': case 'g': return 4;
    case 'T': case 't': return 5;
    default: return 6;
  }
}

}  // namespace

extern "C" sufgpu_status sufgpu_encode_fasta(const char* path, uint8_t* out, uint64_t cap,
                                             uint64_t* size, uint64_t* fingerprint,
                                             uint64_t* records) {
  if (!path || !size) return SUFGPU_INVALID_INPUT;
  gzFile f = gzopen(path, "rb");
  if (!f) return SUFGPU_IO_ERROR;
  Reader r(f);
  std::unordered_set<std::string> names;
  uint64_t written = 0, count = 0, hash = 14695981039346656037ULL;
  auto emit = [&](uint8_t v) {
    if (written < cap && out) out[written] = v;
    ++written;
    hash ^= v;
    hash *= 1099511628211ULL;
  };
  sufgpu_status status = SUFGPU_OK;
  int c = 0;
  // Skip to the first header.
  while ((c = r.get()) >= 0 && c != '>' && c != '@') {
  }
  while (c >= 0 && status == SUFGPU_OK) {
    Record rec;
    // Name: up to the first isspace byte.
    int d;
    while ((d = r.get()) >= 0 && !std::isspace(d)) rec.name.push_back(static_cast<char>(d));
    if (d == -3) { status = SUFGPU_INVALID_INPUT; break; }
    if (d == -1 && rec.name.empty()) break;  // a bare header byte at end of input
    if (d >= 0 && d != '\n') {
      std::string description;
      if (read_line(r, description) < 0) { status = SUFGPU_INVALID_INPUT; break; }
    }
    // Sequence lines.
    while ((c = r.get()) >= 0 && c != '>' && c != '+' && c != '@') {
      if (c == '\n') continue;
      rec.seq.push_back(static_cast<char>(c));
      if (read_line(r, rec.seq) < 0) { c = -3; break; }
      if (rec.seq.size() > 1 && rec.seq.back() == '\r') rec.seq.pop_back();
    }
    if (c == -3) { status = SUFGPU_INVALID_INPUT; break; }
    if (c == '+') {
      // FASTQ: skip the '+' line, then quality lines up to the sequence length.
      int e;
      while ((e = r.get()) >= 0 && e != '\n') {
      }
      if (e < 0) { status = SUFGPU_INVALID_INPUT; break; }
      std::string qual;
      while (qual.size() < rec.seq.size()) {
        std::string line;
        int g = r.get();
        if (g < 0) break;
        if (g != '\n') {
          line.push_back(static_cast<char>(g));
          if (read_line(r, line) < 0) break;
        }
        qual += line;
        if (qual.size() > 1 && qual.back() == '\r') qual.pop_back();
      }
      if (qual.size() != rec.seq.size()) { status = SUFGPU_INVALID_INPUT; break; }
      // The next record starts at the next header byte.
      while ((c = r.get()) >= 0 && c != '>' && c != '@') {
      }
    }
    if (rec.name.empty() || rec.seq.empty() || !names.insert(rec.name).second) {
      status = SUFGPU_INVALID_INPUT;
      break;
    }
    for (const char b : rec.seq) emit(encode_base(static_cast<unsigned char>(b)));
    emit(1);
    ++count;
  }
  gzclose(f);
  if (status == SUFGPU_OK && count == 0) status = SUFGPU_INVALID_INPUT;
  *size = written;
  if (fingerprint) *fingerprint = hash;
  if (records) *records = count;
  return status;
}
