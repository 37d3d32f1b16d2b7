// TEST INFRASTRUCTURE: boost::shared_ptr stand-in (std::shared_ptr) for the reference build.
#ifndef ORACLE_REFSHIM_BOOST_SHARED_PTR
#define ORACLE_REFSHIM_BOOST_SHARED_PTR
#include <memory>
namespace boost {
using std::shared_ptr;
using std::make_shared;
using std::dynamic_pointer_cast;
}
#endif
