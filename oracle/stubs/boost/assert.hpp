/* Stand-in for <boost/assert.hpp> (oracle build scaffolding only). */
#ifndef ORACLE_STUB_BOOST_ASSERT_HPP
#define ORACLE_STUB_BOOST_ASSERT_HPP
#include <cassert>
#define BOOST_ASSERT_MSG(expr, msg) assert((expr) && (msg))
#define BOOST_ASSERT(expr) assert(expr)
#endif
