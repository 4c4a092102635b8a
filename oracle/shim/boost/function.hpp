// Build shim for compiling the reference's CPU runtime without Boost.
// The runtime only needs boost::function as a type-erased callable,
// which std::function provides. Test infrastructure only.
#ifndef ORACLE_SHIM_BOOST_FUNCTION_HPP_
#define ORACLE_SHIM_BOOST_FUNCTION_HPP_
#include <functional>
namespace boost {
using std::function;
}
#endif
