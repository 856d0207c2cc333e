// Test infrastructure only: CPU oracle for the sim-trhepd-rheed multislice path.
// Nothing in the product links or executes this code; only tests/, the smoke check
// and bench.py's CPU-baseline leg do.
//
// Fortran file formats used by the reference drivers:
//   * unformatted sequential records with 4-byte length markers (bulkP.b,
//     written by sim-trhepd-rheed/src/bulkio.f90:126-141,173-176 and
//     bulk.f90:122, read by surfio.f90:99-120,296-304 and surflf.f90:65-72);
//   * list-directed text input (bulk.txt read at bulkio.f90:34-113,
//     surf.txt read at surfio.f90:125-195);
//   * Ew.d formatted output (surflf.f90:162, surfio.f90:270-288).
#pragma once
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace oracle {

using cplx = std::complex<double>;

// ---------------------------------------------------------------- unformatted
class RecordReader {
 public:
  explicit RecordReader(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf_.resize(n);
    if (n && std::fread(buf_.data(), 1, n, f) != (size_t)n) {
      std::fclose(f);
      throw std::runtime_error("short read " + path);
    }
    std::fclose(f);
  }
  // Advance to the next record; subsequent get<T>() calls consume its payload.
  void next() {
    if (pos_ + 4 > buf_.size()) throw std::runtime_error("bulk file: unexpected end");
    int32_t len;
    std::memcpy(&len, &buf_[pos_], 4);
    rec_begin_ = pos_ + 4;
    rec_end_ = rec_begin_ + (size_t)len;
    if (rec_end_ + 4 > buf_.size()) throw std::runtime_error("bulk file: truncated record");
    cur_ = rec_begin_;
    pos_ = rec_end_ + 4;
  }
  template <class T>
  T get() {
    if (cur_ + sizeof(T) > rec_end_) throw std::runtime_error("bulk file: record too short");
    T v;
    std::memcpy(&v, &buf_[cur_], sizeof(T));
    cur_ += sizeof(T);
    return v;
  }
  bool at_end() const { return pos_ >= buf_.size(); }

 private:
  std::vector<unsigned char> buf_;
  size_t pos_ = 0, rec_begin_ = 0, rec_end_ = 0, cur_ = 0;
};

class RecordWriter {
 public:
  explicit RecordWriter(const std::string& path) {
    f_ = std::fopen(path.c_str(), "wb");
    if (!f_) throw std::runtime_error("cannot create " + path);
  }
  ~RecordWriter() {
    if (f_) std::fclose(f_);
  }
  template <class T>
  void put(T v) {
    unsigned char b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    rec_.insert(rec_.end(), b, b + sizeof(T));
  }
  void end_record() {
    int32_t len = (int32_t)rec_.size();
    std::fwrite(&len, 4, 1, f_);
    if (!rec_.empty()) std::fwrite(rec_.data(), 1, rec_.size(), f_);
    std::fwrite(&len, 4, 1, f_);
    rec_.clear();
  }

 private:
  FILE* f_ = nullptr;
  std::vector<unsigned char> rec_;
};

// ---------------------------------------------------------------- list-directed
// A READ statement consumes whole lines until it has its items; the remainder of
// the last line it touched is discarded (that is where the input files keep
// their ",NH,NK,..." annotations).
class ListReader {
 public:
  explicit ListReader(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) throw std::runtime_error("cannot open " + path);
    char line[1 << 16];
    while (std::fgets(line, sizeof line, f)) lines_.emplace_back(line);
    std::fclose(f);
  }
  std::vector<std::string> read(size_t n) {
    std::vector<std::string> out;
    while (out.size() < n) {
      if (li_ >= lines_.size()) throw std::runtime_error("input file: unexpected end");
      const std::string& s = lines_[li_++];
      size_t i = 0;
      while (i < s.size() && out.size() < n) {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r' || s[i] == '\n')) ++i;
        if (i >= s.size()) break;
        if (s[i] == ',') {  // separator (a leading comma after whitespace is consumed)
          ++i;
          continue;
        }
        size_t j = i;
        while (j < s.size() && s[j] != ',' && s[j] != ' ' && s[j] != '\t' && s[j] != '\r' &&
               s[j] != '\n')
          ++j;
        out.push_back(s.substr(i, j - i));
        i = j;
        // swallow one comma that terminates this value
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
        if (i < s.size() && s[i] == ',') ++i;
      }
    }
    return out;
  }
  std::vector<int> ints(size_t n) {
    auto t = read(n);
    std::vector<int> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (int)std::stol(t[i]);
    return v;
  }
  std::vector<double> reals(size_t n) {
    auto t = read(n);
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = to_real(t[i]);
    return v;
  }
  static double to_real(std::string s) {
    for (auto& c : s)
      if (c == 'd' || c == 'D') c = 'e';
    return std::stod(s);
  }

 private:
  std::vector<std::string> lines_;
  size_t li_ = 0;
};

// ---------------------------------------------------------------- formatted out
// Fortran Ew.d edit descriptor: "0.ddddE+xx" right-justified in w columns.
// Exponents beyond two digits drop the 'E' ("0.ddd-100"), as gfortran does.
inline std::string fortran_E(double v, int w, int d) {
  char digits[64];
  std::string mant;
  int exp10 = 0;
  bool neg = std::signbit(v) && v != 0.0;
  double a = std::fabs(v);
  if (a == 0.0) {
    mant = std::string(d, '0');
    exp10 = 0;
  } else {
    std::snprintf(digits, sizeof digits, "%.*e", d - 1, a);  // d.ddd e+XX
    std::string s(digits);
    size_t epos = s.find('e');
    mant = s.substr(0, 1) + s.substr(2, epos - 2);
    exp10 = std::atoi(s.c_str() + epos + 1) + 1;
  }
  char ebuf[16];
  if (std::abs(exp10) <= 99)
    std::snprintf(ebuf, sizeof ebuf, "E%c%02d", exp10 < 0 ? '-' : '+', std::abs(exp10));
  else
    std::snprintf(ebuf, sizeof ebuf, "%c%03d", exp10 < 0 ? '-' : '+', std::abs(exp10));
  std::string body = std::string(neg ? "-" : "") + "0." + mant + ebuf;
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

}  // namespace oracle
