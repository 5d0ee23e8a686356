/* Stand-in for boost::tuple over std::tuple.  ORACLE INFRASTRUCTURE ONLY. */
#ifndef FF_ORACLE_SHIM_BOOST_TUPLE_HPP
#define FF_ORACLE_SHIM_BOOST_TUPLE_HPP
#include <tuple>
namespace boost {
using std::get;
using std::make_tuple;
using std::tuple;
}  // namespace boost
#endif
