// element_groups.cpp -- the material-group block of a BETA input deck
// (BasicModel::ProcessSetElementProperty, BasicModel.cpp:682-775, command
// setElementMaterial / selectElementMaterial / readMaterialGroup()), host only.
//
// The block's lines, read like getLineAndTokenize does (tokens split by
// blanks and tabs, // and /* */ comments removed, blank lines skipped), are
//   first last increment group     elements first, first+increment, ... <= last
//   all group                      every element
// and the block ends at a line whose first token is "end" (any case) or
// whose first number is negative.  Two deliberate departures, both where the
// reference has no defined result: a line of 2 or 3 tokens that is not
// "all" is refused (the reference reads last and increment uninitialised),
// and last must be below the element count (the reference accepts
// last == numElements and writes one element past its array).
#include "../../include/beta_gpu.h"

#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

bool same_nocase(const std::string& a, const char* b) {
  size_t i = 0;
  for (; i < a.size() && b[i]; ++i)
    if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
  return i == a.size() && b[i] == 0;
}

bool to_int(const std::string& t, long long& v) {
  if (t.empty()) return false;
  char* end = nullptr;
  errno = 0;
  v = std::strtoll(t.c_str(), &end, 10);
  return errno == 0 && end && *end == 0;
}

}  // namespace

extern "C" int beta_gpu_parse_element_groups(const char* text, int nelem, int* elem_group, int* nlines) {
  if (!text || nelem <= 0 || !elem_group) return BETA_GPU_ERR_ARG;
  if (nlines) *nlines = 0;
  // comments out, line by line ("/* */" may span lines)
  std::vector<std::vector<std::string>> lines;
  {
    std::vector<std::string> tok;
    std::string cur;
    bool in_block = false;
    auto flush_tok = [&]() {
      if (!cur.empty()) tok.push_back(cur);
      cur.clear();
    };
    for (const char* p = text;; ++p) {
      const char ch = *p;
      if (ch == 0 || ch == '\n') {
        flush_tok();
        if (!tok.empty()) lines.push_back(tok);
        tok.clear();
        if (ch == 0) break;
        continue;
      }
      if (in_block) {
        if (ch == '*' && p[1] == '/') { in_block = false; ++p; }
        continue;
      }
      if (ch == '/' && p[1] == '*') { flush_tok(); in_block = true; ++p; continue; }
      if (ch == '/' && p[1] == '/') {  // to the end of the line
        while (p[1] && p[1] != '\n') ++p;
        continue;
      }
      if (ch == ' ' || ch == '\t' || ch == '\r') flush_tok();
      else cur.push_back(ch);
    }
    if (in_block) return BETA_GPU_ERR_ARG;  // unpaired "/*"
  }
  std::vector<int> out(elem_group, elem_group + nelem);
  int applied = 0;
  for (const auto& t : lines) {
    if (same_nocase(t[0], "end")) break;
    long long first, last, inc, group;
    if (t.size() >= 2 && same_nocase(t[0], "all")) {
      first = 0;
      last = nelem - 1;
      inc = 1;
      if (!to_int(t[1], group)) return BETA_GPU_ERR_ARG;
    } else {
      if (!to_int(t[0], first)) return BETA_GPU_ERR_ARG;
      if (first < 0) break;  // a negative element number ends the block
      if (t.size() < 4 || !to_int(t[1], last) || !to_int(t[2], inc) || !to_int(t[3], group))
        return BETA_GPU_ERR_ARG;
    }
    if (first > last || last >= nelem || inc < 1 || group < 0 || group > 2147483647LL) return BETA_GPU_ERR_ARG;
    for (long long e = first; e <= last; e += inc) out[e] = (int)group;
    ++applied;
  }
  for (int e = 0; e < nelem; ++e) elem_group[e] = out[e];
  if (nlines) *nlines = applied;
  return BETA_GPU_OK;
}
