// Shim: the ascending, duplicate-free list the reference's sparse storage
// keeps per row (SortedList<T> as sparse.cpp uses it: add, find -- the index
// or getNum() when absent --, getNum, [], binary I/O and print), written for
// this build because the reference ships no headers.
#pragma once
#include <algorithm>
#include <cstdio>
#include <iostream>
#include <vector>

template <class T>
class SortedList {
 public:
  void add(const T& v) {
    auto it = std::lower_bound(d_.begin(), d_.end(), v);
    if (it == d_.end() || *it != v) d_.insert(it, v);
  }
  int find(const T& v) const {
    auto it = std::lower_bound(d_.begin(), d_.end(), v);
    return (it != d_.end() && *it == v) ? (int)(it - d_.begin()) : (int)d_.size();
  }
  int getNum() const { return (int)d_.size(); }
  const T& operator[](int i) const { return d_[i]; }
  void fwrite(FILE* f) const {
    int n = (int)d_.size();
    std::fwrite(&n, sizeof(int), 1, f);
    if (n) std::fwrite(d_.data(), sizeof(T), n, f);
  }
  void fread(FILE* f) {
    int n = 0;
    if (std::fread(&n, sizeof(int), 1, f) != 1) n = 0;
    d_.resize(n);
    if (n && std::fread(d_.data(), sizeof(T), n, f) != (size_t)n) d_.clear();
  }
  std::ostream& print(std::ostream& os) const {
    for (const T& v : d_) os << ' ' << v;
    return os;
  }

 private:
  std::vector<T> d_;
};
