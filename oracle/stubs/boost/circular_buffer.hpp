/* Empty stand-in: included by reference headers, unused on the oracle path. */
#ifndef ORACLE_STUB_BOOST_CIRCULAR_BUFFER_HPP
#define ORACLE_STUB_BOOST_CIRCULAR_BUFFER_HPP
#endif
