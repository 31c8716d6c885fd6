/*
 * Test-infrastructure stand-in for <boost/thread/barrier.hpp> on the C++11
 * standard library.  barrier(n).wait() blocks until n threads have called it,
 * then releases them all and re-arms for the next round; exactly one of the
 * released threads (the last to arrive) gets true, as Boost's does.
 */
#ifndef GZ_REFSTUB_BOOST_THREAD_BARRIER_HPP_
#define GZ_REFSTUB_BOOST_THREAD_BARRIER_HPP_
#include <condition_variable>
#include <mutex>

namespace boost {

class barrier {
 public:
  explicit barrier(unsigned int count)
      : threshold_(count), waiting_(0), generation_(0) {}

  bool wait() {
    std::unique_lock<std::mutex> lock(m_);
    const unsigned long arrival_generation = generation_;
    if (++waiting_ == threshold_) {
      waiting_ = 0;
      ++generation_;
      released_.notify_all();
      return true;
    }
    while (generation_ == arrival_generation) released_.wait(lock);
    return false;
  }

 private:
  barrier(const barrier &);
  barrier &operator=(const barrier &);

  std::mutex m_;
  std::condition_variable released_;
  const unsigned int threshold_;
  unsigned int waiting_;
  unsigned long generation_;
};

}  // namespace boost
#endif
