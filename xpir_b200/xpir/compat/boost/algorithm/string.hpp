// Minimal stand-in for boost::algorithm::split / is_any_of, enough for the XPIR
// reference sources that parse "LWE:k:N:logq" descriptors.
#ifndef XPIR_REF_SHIM_BOOST_ALGORITHM_STRING_HPP
#define XPIR_REF_SHIM_BOOST_ALGORITHM_STRING_HPP

#include <string>
#include <vector>

namespace boost {
namespace algorithm {

struct is_any_of_pred {
  std::string set;
  bool operator()(char c) const { return set.find(c) != std::string::npos; }
};

inline is_any_of_pred is_any_of(const std::string &s) { return is_any_of_pred{s}; }
inline is_any_of_pred is_any_of(const char *s) { return is_any_of_pred{std::string(s)}; }

// Token-compress-off semantics: every separator ends a token, so adjacent separators
// give empty tokens and the result always has (#separators + 1) entries.
template <class Seq>
Seq &split(Seq &out, const std::string &in, const is_any_of_pred &pred) {
  out.clear();
  std::string cur;
  for (char c : in) {
    if (pred(c)) {
      out.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(c);
    }
  }
  out.push_back(cur);
  return out;
}

}  // namespace algorithm
using algorithm::is_any_of;
using algorithm::split;
}  // namespace boost

#endif
