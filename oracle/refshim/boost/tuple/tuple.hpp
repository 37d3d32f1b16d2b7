// TEST INFRASTRUCTURE: boost::tuple stand-in (std::tuple) for the reference build.
#ifndef ORACLE_REFSHIM_BOOST_TUPLE
#define ORACLE_REFSHIM_BOOST_TUPLE
#include <tuple>
namespace boost {
template<typename... T> using tuple = std::tuple<T...>;
using std::make_tuple;
using std::get;
namespace tuples {
template<typename... T> using tuple = std::tuple<T...>;
using std::make_tuple;
using std::get;
}
}
#endif
