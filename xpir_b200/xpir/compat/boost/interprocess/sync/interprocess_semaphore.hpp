// Minimal pthread-based stand-in for boost::interprocess::interprocess_semaphore, as
// used by XPIR's shared_queue.
#ifndef XPIR_REF_SHIM_INTERPROCESS_SEMAPHORE_HPP
#define XPIR_REF_SHIM_INTERPROCESS_SEMAPHORE_HPP

#include <pthread.h>

namespace boost {
namespace interprocess {

class interprocess_semaphore {
 public:
  explicit interprocess_semaphore(unsigned int initial) : count_(initial) {
    pthread_mutex_init(&m_, nullptr);
    pthread_cond_init(&c_, nullptr);
  }
  ~interprocess_semaphore() {
    pthread_cond_destroy(&c_);
    pthread_mutex_destroy(&m_);
  }
  void post() {
    pthread_mutex_lock(&m_);
    ++count_;
    pthread_cond_signal(&c_);
    pthread_mutex_unlock(&m_);
  }
  void wait() {
    pthread_mutex_lock(&m_);
    while (count_ == 0) pthread_cond_wait(&c_, &m_);
    --count_;
    pthread_mutex_unlock(&m_);
  }
  bool try_wait() {
    pthread_mutex_lock(&m_);
    bool ok = count_ > 0;
    if (ok) --count_;
    pthread_mutex_unlock(&m_);
    return ok;
  }

 private:
  unsigned long count_;
  pthread_mutex_t m_;
  pthread_cond_t c_;
};

}  // namespace interprocess
}  // namespace boost

#endif
