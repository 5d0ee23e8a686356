/* Stand-in for boost/tuple/tuple_comparison.hpp.  ORACLE INFRASTRUCTURE ONLY. */
#include "tuple.hpp"
