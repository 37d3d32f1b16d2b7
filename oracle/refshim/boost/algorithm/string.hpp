// TEST INFRASTRUCTURE: boost::split / boost::is_any_of stand-ins for the
// reference build (StateBase splits "field|nodelist" keys with them).
#ifndef ORACLE_REFSHIM_BOOST_STRING
#define ORACLE_REFSHIM_BOOST_STRING
#include <string>
namespace boost {
struct is_any_of_pred {
  std::string chars;
  bool operator()(char c) const { return chars.find(c) != std::string::npos; }
};
inline is_any_of_pred is_any_of(const std::string& s) { return is_any_of_pred{s}; }
template<class Seq> Seq& split(Seq& out, const std::string& in, const is_any_of_pred& pred) {
  out.clear();
  std::string cur;
  for (char c : in) {
    if (pred(c)) { out.push_back(cur); cur.clear(); }
    else cur.push_back(c);
  }
  out.push_back(cur);
  return out;
}
}
#endif
