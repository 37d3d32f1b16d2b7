// TEST INFRASTRUCTURE: boost::hash stand-in for the reference build (the
// Mesh headers name it; nothing on the checked path hashes).
#ifndef ORACLE_REFSHIM_BOOST_HASH
#define ORACLE_REFSHIM_BOOST_HASH
#include <cstddef>
#include <functional>
namespace boost {
template<class T> struct hash : std::hash<T> {};
template<class T> inline void hash_combine(std::size_t& seed, const T& v) {
  seed ^= std::hash<T>()(v) + 0x9e3779b9 + (seed << 6) + (seed >> 2);
}
}
#endif
