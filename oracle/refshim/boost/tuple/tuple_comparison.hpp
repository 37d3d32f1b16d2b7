// TEST INFRASTRUCTURE: std::tuple compares already; nothing more is needed.
#ifndef ORACLE_REFSHIM_BOOST_TUPLE_COMPARISON
#define ORACLE_REFSHIM_BOOST_TUPLE_COMPARISON
#include "boost/tuple/tuple.hpp"
#endif
