// Build shim for compiling the reference's CPU runtime without Boost.
// The runtime derives from boost::array and calls assign(v), the Boost
// name for filling every element. Test infrastructure only.
#ifndef ORACLE_SHIM_BOOST_ARRAY_HPP_
#define ORACLE_SHIM_BOOST_ARRAY_HPP_
#include <array>
#include <cstddef>
namespace boost {
template <class T, std::size_t N>
struct array : public std::array<T, N> {
  void assign(const T &v) { this->fill(v); }
};
}
#endif
