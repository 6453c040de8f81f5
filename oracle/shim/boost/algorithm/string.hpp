// Minimal stand-in for the three Boost string algorithms the feMorph
// reference uses in its .dat reader (trim, split on a character set with
// token compression, to_upper_copy).  Written for this project; it is only
// used to compile the reference as a CPU oracle.
#pragma once
#include <algorithm>
#include <cctype>
#include <string>
#include <vector>
namespace boost {
enum token_compress_mode_type { token_compress_on, token_compress_off };
struct fm_char_set { std::string chars; };
inline fm_char_set is_any_of(const char* s) { return fm_char_set{s}; }
inline void trim(std::string& s) {
  size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b])) ++b;
  while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
  s = s.substr(b, e - b);
}
inline std::string to_upper_copy(const std::string& s) {
  std::string r(s);
  for (auto& c : r) c = (char)std::toupper((unsigned char)c);
  return r;
}
// Splits s at any character of set.  With token_compress_on, adjacent
// separators produce one split (an empty leading/trailing token is kept,
// as Boost does).
inline std::vector<std::string>& split(std::vector<std::string>& out, const std::string& s,
                                       const fm_char_set& set, token_compress_mode_type mode = token_compress_off) {
  out.clear();
  std::string cur;
  size_t i = 0, n = s.size();
  while (i < n) {
    if (set.chars.find(s[i]) != std::string::npos) {
      out.push_back(cur);
      cur.clear();
      ++i;
      if (mode == token_compress_on)
        while (i < n && set.chars.find(s[i]) != std::string::npos) ++i;
    } else {
      cur.push_back(s[i++]);
    }
  }
  out.push_back(cur);
  return out;
}
}  // namespace boost
