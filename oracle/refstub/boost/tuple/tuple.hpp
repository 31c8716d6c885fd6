/*
 * Test-infrastructure stand-in for <boost/tuple/tuple.hpp>: the reference
 * includes it (src/extension_seed_list.h) but names nothing from it.
 */
#ifndef GZ_REFSTUB_BOOST_TUPLE_TUPLE_HPP_
#define GZ_REFSTUB_BOOST_TUPLE_TUPLE_HPP_
#endif
