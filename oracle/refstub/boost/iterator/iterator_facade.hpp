/*
 * Test-infrastructure stand-in for <boost/iterator/iterator_facade.hpp>: the
 * reference includes it (src/extension_seed_list.h) but names nothing from it.
 */
#ifndef GZ_REFSTUB_BOOST_ITERATOR_FACADE_HPP_
#define GZ_REFSTUB_BOOST_ITERATOR_FACADE_HPP_
#endif
