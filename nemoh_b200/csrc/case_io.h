// Reading the reference's text case files the way its Fortran list-directed
// READ does: every read starts a new record (line) and takes as many values as
// asked for, continuing on the following lines if needed; the rest of the last
// line is dropped. '!' starts a comment; ',' and tabs separate values.
#pragma once
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace nb200io {

struct IoError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class Records {
 public:
  explicit Records(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw IoError("cannot open " + path);
    std::string s;
    while (std::getline(f, s)) lines_.push_back(s);
  }
  // skip one record (a READ with an empty list)
  void skip() { ++pos_; }
  std::vector<std::string> read(size_t n) {
    std::vector<std::string> v;
    if (n == 0) {
      skip();
      return v;
    }
    while (v.size() < n) {
      if (pos_ >= lines_.size()) throw IoError("unexpected end of file");
      std::string s = lines_[pos_++];
      const size_t bang = s.find('!');
      if (bang != std::string::npos) s.resize(bang);
      for (char& ch : s)
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      std::istringstream is(s);
      std::string t;
      while (is >> t) v.push_back(t);
    }
    v.resize(n);
    return v;
  }
  double real() { return std::stod(read(1)[0]); }
  int integer() { return std::stoi(read(1)[0]); }
  // raw text of the next record (for section markers)
  bool next_line(std::string& s) {
    if (pos_ >= lines_.size()) return false;
    s = lines_[pos_++];
    return true;
  }

 private:
  std::vector<std::string> lines_;
  size_t pos_ = 0;
};

// <root>/ID.dat (Common/Identification.f90:30-37): the case directory
inline std::string case_dir(const std::string& root) {
  const std::string pre = root.empty() ? "" : root + "/";
  Records idr(pre + "ID.dat");
  const int lid = idr.integer();
  return pre + idr.read(1)[0].substr(0, lid);
}

}  // namespace nb200io
