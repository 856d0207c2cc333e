// Readers for the reference's Fortran file formats and the form-factor lookup,
// shared by the surface and bulk host models.
#pragma once
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "scattering_tables.h"

namespace trhepd {
namespace ftext {

// ------------------------------------------------------------ unformatted records
class Records {
 public:
  explicit Records(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    data_.resize(n > 0 ? n : 0);
    if (n > 0 && std::fread(data_.data(), 1, n, f) != (size_t)n) {
      std::fclose(f);
      throw std::runtime_error("short read " + path);
    }
    std::fclose(f);
  }
  void begin() {
    if (at_ + 4 > data_.size()) throw std::runtime_error("bulkP.b: missing record");
    int32_t len;
    std::memcpy(&len, &data_[at_], 4);
    if (len < 0 || at_ + 8 + (size_t)len > data_.size())
      throw std::runtime_error("bulkP.b: bad record length");
    cur_ = at_ + 4;
    end_ = cur_ + len;
    at_ = end_ + 4;
  }
  int32_t i4() { return take<int32_t>(); }
  double r8() { return take<double>(); }

 private:
  template <class T>
  T take() {
    if (cur_ + sizeof(T) > end_) throw std::runtime_error("bulkP.b: record too short");
    T v;
    std::memcpy(&v, &data_[cur_], sizeof(T));
    cur_ += sizeof(T);
    return v;
  }
  std::vector<unsigned char> data_;
  size_t at_ = 0, cur_ = 0, end_ = 0;
};

// ------------------------------------------------------------ list-directed text
class ListInput {
 public:
  explicit ListInput(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) throw std::runtime_error("cannot open " + path);
    std::string line;
    int c;
    while ((c = std::fgetc(f)) != EOF) {
      if (c == '\n') {
        lines_.push_back(line);
        line.clear();
      } else {
        line.push_back((char)c);
      }
    }
    if (!line.empty()) lines_.push_back(line);
    std::fclose(f);
  }
  // One READ statement: consume lines until n values are collected; the rest of the
  // last line is ignored (that is where the files keep their annotations).
  std::vector<std::string> values(size_t n) {
    std::vector<std::string> out;
    while (out.size() < n) {
      if (next_ >= lines_.size()) throw std::runtime_error("input ended early");
      const std::string& s = lines_[next_++];
      size_t i = 0;
      while (i < s.size() && out.size() < n) {
        char ch = s[i];
        if (ch == ' ' || ch == '\t' || ch == '\r' || ch == ',') {
          ++i;
          continue;
        }
        size_t j = i;
        while (j < s.size() && s[j] != ',' && s[j] != ' ' && s[j] != '\t' && s[j] != '\r') ++j;
        out.push_back(s.substr(i, j - i));
        i = j;
      }
    }
    return out;
  }
  int integer() { return std::stoi(values(1)[0]); }
  static double real(std::string s) {
    for (char& ch : s)
      if (ch == 'd' || ch == 'D') ch = 'e';
    return std::stod(s);
  }

 private:
  std::vector<std::string> lines_;
  size_t next_ = 0;
};

// ------------------------------------------------------------ form factors
inline int form_factor_params(int iz, int iabr, double* a, double* b) {  // asf.f90:415-431
  if (iz < 1 || iz > 98) return 0;
  const double* row = (iabr == 0 && trhepd_tables::kDoyleTurner[iz - 1][0] > 1e-5)
                          ? trhepd_tables::kDoyleTurner[iz - 1]
                          : trhepd_tables::kPeng[iz - 1];
  for (int i = 0; i < 4; ++i) {
    a[i] = row[i];
    b[i] = row[4 + i];
  }
  return 4;
}


inline double atomic_mass(int iz) {
  return (iz >= 1 && iz <= 110) ? trhepd_tables::kAtomicMass[iz - 1] : 1000.0;
}

}  // namespace ftext
}  // namespace trhepd
