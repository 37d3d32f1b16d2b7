// TEST INFRASTRUCTURE: boost::static_assert stand-in for the reference build.
#ifndef ORACLE_REFSHIM_BOOST_STATIC_ASSERT
#define ORACLE_REFSHIM_BOOST_STATIC_ASSERT
#define BOOST_STATIC_ASSERT(x) static_assert((x), #x)
#endif
