// Minimal pthread-based stand-in for the boost::thread / boost::mutex subset that the
// XPIR reference sources use.  It deliberately avoids
// <thread> and <mutex>: the reference headers say "using namespace std; using namespace
// boost;" and then name `thread` unqualified, so std::thread must not be visible.
#ifndef XPIR_REF_SHIM_BOOST_THREAD_HPP
#define XPIR_REF_SHIM_BOOST_THREAD_HPP

#include <pthread.h>
#include <sched.h>
#include <time.h>

#include <functional>
#include <utility>

namespace boost {

class mutex {
 public:
  mutex() { pthread_mutex_init(&m_, nullptr); }
  ~mutex() { pthread_mutex_destroy(&m_); }
  mutex(const mutex &) = delete;
  mutex &operator=(const mutex &) = delete;
  void lock() { pthread_mutex_lock(&m_); }
  void unlock() { pthread_mutex_unlock(&m_); }
  bool try_lock() { return pthread_mutex_trylock(&m_) == 0; }

  class scoped_lock {
   public:
    explicit scoped_lock(mutex &m) : m_(m) { m_.lock(); }
    ~scoped_lock() { m_.unlock(); }
    scoped_lock(const scoped_lock &) = delete;
    scoped_lock &operator=(const scoped_lock &) = delete;

   private:
    mutex &m_;
  };

 private:
  pthread_mutex_t m_;
};

class recursive_mutex {
 public:
  recursive_mutex() {
    pthread_mutexattr_t a;
    pthread_mutexattr_init(&a);
    pthread_mutexattr_settype(&a, PTHREAD_MUTEX_RECURSIVE);
    pthread_mutex_init(&m_, &a);
    pthread_mutexattr_destroy(&a);
  }
  ~recursive_mutex() { pthread_mutex_destroy(&m_); }
  void lock() { pthread_mutex_lock(&m_); }
  void unlock() { pthread_mutex_unlock(&m_); }
  bool try_lock() { return pthread_mutex_trylock(&m_) == 0; }

 private:
  pthread_mutex_t m_;
};

class thread {
 public:
  thread() = default;
  template <class F, class... Args>
  explicit thread(F &&f, Args &&...args) {
    auto *fn = new std::function<void()>(std::bind(std::forward<F>(f), std::forward<Args>(args)...));
    if (pthread_create(&tid_, nullptr, &thread::trampoline, fn) == 0) {
      running_ = true;
    } else {
      delete fn;
    }
  }
  thread(thread &&o) noexcept : tid_(o.tid_), running_(o.running_) { o.running_ = false; }
  thread &operator=(thread &&o) noexcept {
    if (running_) join();
    tid_ = o.tid_;
    running_ = o.running_;
    o.running_ = false;
    return *this;
  }
  thread(const thread &) = delete;
  thread &operator=(const thread &) = delete;
  ~thread() {
    if (running_) pthread_detach(tid_);
  }
  bool joinable() const { return running_; }
  void join() {
    if (running_) {
      pthread_join(tid_, nullptr);
      running_ = false;
    }
  }

 private:
  static void *trampoline(void *p) {
    auto *fn = static_cast<std::function<void()> *>(p);
    (*fn)();
    delete fn;
    return nullptr;
  }
  pthread_t tid_{};
  bool running_ = false;
};

namespace posix_time {
struct milliseconds {
  explicit milliseconds(long v) : ms(v) {}
  long ms;
};
}  // namespace posix_time

namespace this_thread {
inline void sleep(const posix_time::milliseconds &d) {
  struct timespec ts;
  ts.tv_sec = d.ms / 1000;
  ts.tv_nsec = (d.ms % 1000) * 1000000L;
  nanosleep(&ts, nullptr);
}
inline void yield() { sched_yield(); }
}  // namespace this_thread

}  // namespace boost

#endif
