// Shim: the report writer Equations prints through -- headings and stream
// insertion onto one output stream.
#pragma once
#include <iostream>

class FormWriter {
 public:
  explicit FormWriter(std::ostream* os = &std::cout) : os_(os) {}
  void h2(const char* title) { *os_ << "== " << title << " ==\n"; }
  std::ostream* getOutputStream() { return os_; }
  template <class T>
  FormWriter& operator<<(const T& v) {
    *os_ << v;
    return *this;
  }
  FormWriter& operator<<(std::ostream& (*manip)(std::ostream&)) {
    *os_ << manip;
    return *this;
  }

 private:
  std::ostream* os_;
};
