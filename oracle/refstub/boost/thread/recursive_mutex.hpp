/*
 * Test-infrastructure stand-in for <boost/thread/recursive_mutex.hpp> on the
 * C++11 standard library (boost::recursive_mutex and its scoped_lock).
 */
#ifndef GZ_REFSTUB_BOOST_THREAD_RECURSIVE_MUTEX_HPP_
#define GZ_REFSTUB_BOOST_THREAD_RECURSIVE_MUTEX_HPP_
#include <mutex>

namespace boost {

class recursive_mutex : public std::recursive_mutex {
 public:
  typedef std::unique_lock<std::recursive_mutex> scoped_lock;
};

}  // namespace boost
#endif
