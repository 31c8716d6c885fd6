/*
 * Test-infrastructure stand-in for <boost/thread.hpp> on the C++11 standard
 * library, so that the reference's host sources (which use Boost only for
 * threads, locks, barriers and bind) compile into the oracle's reference
 * build without Boost.  boost::thread wraps std::thread; thread_group owns the
 * threads it creates and joins them in join_all(); boost::bind forwards to
 * std::bind (both copy their bound arguments).
 */
#ifndef GZ_REFSTUB_BOOST_THREAD_HPP_
#define GZ_REFSTUB_BOOST_THREAD_HPP_
#include <functional>
#include <list>
#include <mutex>
#include <thread>
#include <utility>

#include "thread/barrier.hpp"
#include "thread/mutex.hpp"
#include "thread/recursive_mutex.hpp"

namespace boost {

class thread {
 public:
  template <typename F>
  explicit thread(F f) : t_(f) {}
  ~thread() {
    if (t_.joinable()) t_.join();
  }
  void join() {
    if (t_.joinable()) t_.join();
  }
  bool joinable() const { return t_.joinable(); }

 private:
  thread(const thread &);
  thread &operator=(const thread &);
  std::thread t_;
};

class thread_group {
 public:
  thread_group() {}
  ~thread_group() {
    for (std::list<thread *>::iterator it = threads_.begin();
         it != threads_.end(); ++it)
      delete *it;
  }
  template <typename F>
  thread *create_thread(F f) {
    std::lock_guard<std::mutex> lock(m_);
    thread *t = new thread(f);
    threads_.push_back(t);
    return t;
  }
  void join_all() {
    std::lock_guard<std::mutex> lock(m_);
    for (std::list<thread *>::iterator it = threads_.begin();
         it != threads_.end(); ++it)
      (*it)->join();
  }

 private:
  thread_group(const thread_group &);
  thread_group &operator=(const thread_group &);
  std::mutex m_;
  std::list<thread *> threads_;
};

template <typename... Args>
auto bind(Args &&... args)
    -> decltype(std::bind(std::forward<Args>(args)...)) {
  return std::bind(std::forward<Args>(args)...);
}

}  // namespace boost
#endif
