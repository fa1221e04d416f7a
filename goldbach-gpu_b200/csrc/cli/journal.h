// journal.h -- append-only segment journal for resumable range runs.
//
// Extends the reference's `--start=` restart point (src/goldbach.cu:581,
// 689), which restarts a run from a number the user must work out, to a
// journal the verifier keeps itself: one line per batch of completed
// segments, written and fsync'ed as soon as the batch's results are back, so
// a run over [4, 1e12] that is interrupted (power, preemption, a killed job)
// resumes with the same command line and skips every journaled segment.
//
// Format (text, one record per line):
//   goldbach-journal v1 start=S limit=L seg_size=Z p_small=P phase2=Q
//   seg LO HI checked C fallbacks F failures X first_fail N max_minp M sum H
// LO..HI-1 are segment indices of the full range (segment i covers the
// SEG_SIZE even n from START + 2*SEG_SIZE*i); H is the FNV-1a 64 hash (hex)
// of the line's text before " sum ".  A line that is cut short or whose
// hash does not match (a write torn by the interruption) ends the journal:
// the file is truncated there and those segments run again.
#pragma once
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cinttypes>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace gbj {

struct Key {
  uint64_t start, limit, seg_size, p_small, phase2;
};

struct Record {
  uint64_t lo, hi;  // segments [lo, hi)
  uint64_t checked, fallbacks, failures, first_fail, max_minp;
};

inline uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

inline std::string header_line(const Key& k) {
  char buf[256];
  std::snprintf(buf, sizeof buf,
                "goldbach-journal v1 start=%" PRIu64 " limit=%" PRIu64 " seg_size=%" PRIu64
                " p_small=%" PRIu64 " phase2=%" PRIu64,
                k.start, k.limit, k.seg_size, k.p_small, k.phase2);
  return buf;
}

inline std::string record_line(const Record& r) {
  char buf[320];
  std::snprintf(buf, sizeof buf,
                "seg %" PRIu64 " %" PRIu64 " checked %" PRIu64 " fallbacks %" PRIu64
                " failures %" PRIu64 " first_fail %" PRIu64 " max_minp %" PRIu64,
                r.lo, r.hi, r.checked, r.fallbacks, r.failures, r.first_fail, r.max_minp);
  std::string body = buf;
  std::snprintf(buf, sizeof buf, " sum %016" PRIx64, fnv1a(body));
  return body + buf;
}

// Parses one record line; false when it is malformed or its hash differs.
inline bool parse_record(const std::string& line, Record* r) {
  const size_t at = line.rfind(" sum ");
  if (at == std::string::npos) return false;
  const std::string body = line.substr(0, at);
  char want[32];
  std::snprintf(want, sizeof want, "%016" PRIx64, fnv1a(body));
  if (line.substr(at + 5) != want) return false;
  std::istringstream in(body);
  std::string t[7];
  Record x{};
  in >> t[0] >> x.lo >> x.hi >> t[1] >> x.checked >> t[2] >> x.fallbacks >> t[3] >> x.failures >>
      t[4] >> x.first_fail >> t[5] >> x.max_minp;
  if (!in || t[0] != "seg" || t[1] != "checked" || t[2] != "fallbacks" || t[3] != "failures" ||
      t[4] != "first_fail" || t[5] != "max_minp" || x.lo >= x.hi)
    return false;
  *r = x;
  return true;
}

class Journal {
 public:
  // Opens (or creates) the journal for this run.  An existing journal must
  // carry the same key; its good records are loaded and a torn tail is cut.
  bool open(const std::string& path, const Key& key, std::string* err) {
    path_ = path;
    std::ifstream in(path, std::ios::binary);
    if (in) {
      std::string all((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
      size_t pos = 0, good_end = 0;
      bool first = true;
      while (pos < all.size()) {
        const size_t nl = all.find('\n', pos);
        if (nl == std::string::npos) break;  // a line cut short
        const std::string line = all.substr(pos, nl - pos);
        if (first) {
          if (line != header_line(key)) {
            *err = "journal " + path + " belongs to another run (" + line + ")";
            return false;
          }
          first = false;
        } else {
          Record r;
          if (!parse_record(line, &r)) break;
          recs_.push_back(r);
        }
        pos = nl + 1;
        good_end = pos;
      }
      // (no complete header line: the run that created the file was stopped
      // before its first write finished; start the journal afresh)
      if (good_end < all.size()) {
        if (truncate(path.c_str(), (off_t)good_end) != 0) {
          *err = "cannot truncate the torn tail of journal " + path;
          return false;
        }
      }
      if (good_end > 0) return open_append(err);
    }
    if (!open_append(err)) return false;
    return write_line(header_line(key), err);
  }

  bool append(const Record& r, std::string* err) {
    if (!write_line(record_line(r), err)) return false;
    recs_.push_back(r);
    return true;
  }

  const std::vector<Record>& records() const { return recs_; }

  ~Journal() {
    if (fd_ >= 0) close(fd_);
  }

 private:
  bool open_append(std::string* err) {
    fd_ = ::open(path_.c_str(), O_WRONLY | O_CREAT | O_APPEND, 0644);
    if (fd_ < 0) {
      *err = "cannot open journal " + path_;
      return false;
    }
    return true;
  }
  bool write_line(const std::string& line, std::string* err) {
    const std::string s = line + "\n";
    if (::write(fd_, s.data(), s.size()) != (ssize_t)s.size() || fsync(fd_) != 0) {
      *err = "cannot write journal " + path_;
      return false;
    }
    return true;
  }
  std::string path_;
  int fd_ = -1;
  std::vector<Record> recs_;
};

// Segment ranges [lo, hi) of [0, nseg) that no record covers, split into
// batches of at most `per` segments.
inline std::vector<std::pair<uint64_t, uint64_t>> pending_batches(
    const std::vector<Record>& recs, uint64_t nseg, uint64_t per) {
  std::vector<std::pair<uint64_t, uint64_t>> iv, out;
  for (const Record& r : recs) iv.push_back({r.lo, r.hi < nseg ? r.hi : nseg});
  // the complement of the journaled intervals, without one flag per segment
  std::sort(iv.begin(), iv.end());
  uint64_t cur = 0;
  auto emit = [&](uint64_t a, uint64_t b) {
    for (uint64_t x = a; x < b; x += per) out.push_back({x, x + per < b ? x + per : b});
  };
  for (const auto& d : iv) {
    if (d.first > cur) emit(cur, d.first < nseg ? d.first : nseg);
    if (d.second > cur) cur = d.second;
    if (cur >= nseg) break;
  }
  if (cur < nseg) emit(cur, nseg);
  return out;
}

}  // namespace gbj
