/*
 * Test-infrastructure stand-in for <boost/tr1/memory.hpp>: the reference names
 * std::tr1::shared_ptr, which libstdc++ still provides in <tr1/memory>.
 */
#ifndef GZ_REFSTUB_BOOST_TR1_MEMORY_HPP_
#define GZ_REFSTUB_BOOST_TR1_MEMORY_HPP_
#include <tr1/memory>
#endif
