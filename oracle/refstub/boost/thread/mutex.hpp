/*
 * Test-infrastructure stand-in for <boost/thread/mutex.hpp>, built on the C++11
 * standard library.  Only the names the reference's sources use when they are
 * compiled into the oracle's reference build exist here: boost::mutex with its
 * scoped_lock, and boost::unique_lock.
 */
#ifndef GZ_REFSTUB_BOOST_THREAD_MUTEX_HPP_
#define GZ_REFSTUB_BOOST_THREAD_MUTEX_HPP_
#include <mutex>

namespace boost {

class mutex : public std::mutex {
 public:
  typedef std::unique_lock<std::mutex> scoped_lock;
};

template <typename Lockable>
class unique_lock : public std::unique_lock<std::mutex> {
 public:
  explicit unique_lock(Lockable &m) : std::unique_lock<std::mutex>(m) {}
};

}  // namespace boost
#endif
