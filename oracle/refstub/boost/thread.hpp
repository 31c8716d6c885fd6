/*
 * Declaration-only stand-in for <boost/thread.hpp>, used when compiling the
 * reference's arithmetic units into the test-only reference library.  The
 * compiled units only name these types in declarations of pointers and
 * functions that are never called here; nothing is defined, so no Boost
 * behaviour is reproduced.
 */
#ifndef GZ_REFSTUB_BOOST_THREAD_HPP_
#define GZ_REFSTUB_BOOST_THREAD_HPP_
namespace boost {
class mutex;
class barrier;
}
#endif
