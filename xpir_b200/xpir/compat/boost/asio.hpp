// Minimal stand-in for the part of Boost.Asio that XPIR's server, client and optimizer use
// (apps/server, apps/client, apps/optim): blocking TCP sockets over POSIX, the free
// functions read/write on whole buffers, an io_service whose run() executes posted work and
// pending async_accept operations in order, and a signal_set that leaves the default action
// of the signals in place.  It deliberately avoids <thread> and <mutex> (XPIR's headers say
// "using namespace std; using namespace boost;" and name `thread` and `mutex` unqualified).
#ifndef XPIR_COMPAT_BOOST_ASIO_HPP
#define XPIR_COMPAT_BOOST_ASIO_HPP

#include <arpa/inet.h>
#include <errno.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <pthread.h>
#include <string.h>
#include <sys/socket.h>
#include <sys/types.h>
#include <unistd.h>

#include <cstddef>
#include <deque>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include <boost/bind.hpp>

namespace boost {
// boost/cstdint.hpp's names, which XPIR's server spells boost::uint64_t and the like.
using ::int32_t;
using ::int64_t;
using ::uint32_t;
using ::uint64_t;
using ::uint8_t;

namespace system {

class error_code {
 public:
  error_code() : v_(0) {}
  explicit error_code(int v) : v_(v) {}
  int value() const { return v_; }
  explicit operator bool() const { return v_ != 0; }
  bool operator!() const { return v_ == 0; }
  std::string message() const { return v_ ? std::string(strerror(v_)) : std::string("Success"); }

 private:
  int v_;
};

class system_error : public std::runtime_error {
 public:
  explicit system_error(const error_code &e, const std::string &what = "")
      : std::runtime_error(what.empty() ? e.message() : what + ": " + e.message()), code_(e) {}
  const error_code &code() const { return code_; }

 private:
  error_code code_;
};

}  // namespace system

namespace asio {

// ---- buffers -------------------------------------------------------------------------
struct mutable_buffer {
  void *data;
  std::size_t size;
};
struct const_buffer {
  const void *data;
  std::size_t size;
  const_buffer(const void *d, std::size_t n) : data(d), size(n) {}
  const_buffer(const mutable_buffer &b) : data(b.data), size(b.size) {}
};
inline mutable_buffer buffer(void *d, std::size_t n) { return mutable_buffer{d, n}; }
inline const_buffer buffer(const void *d, std::size_t n) { return const_buffer(d, n); }
inline const_buffer buffer(const std::string &s) { return const_buffer(s.data(), s.size()); }
template <class T>
inline mutable_buffer buffer(std::vector<T> &v) { return mutable_buffer{v.data(), v.size() * sizeof(T)}; }

// ---- io_service ------------------------------------------------------------------------
class io_service {
 public:
  io_service() : stopped_(false) {
    pthread_mutex_init(&mu_, nullptr);
    pthread_cond_init(&cv_, nullptr);
  }
  ~io_service() {
    pthread_cond_destroy(&cv_);
    pthread_mutex_destroy(&mu_);
  }
  io_service(const io_service &) = delete;
  io_service &operator=(const io_service &) = delete;

  void post(std::function<void()> f) {
    pthread_mutex_lock(&mu_);
    work_.push_back(std::move(f));
    pthread_cond_signal(&cv_);
    pthread_mutex_unlock(&mu_);
  }
  // Runs queued work in order until stop() or until nothing is left.
  std::size_t run() {
    std::size_t n = 0;
    for (;;) {
      pthread_mutex_lock(&mu_);
      if (stopped_ || work_.empty()) {
        pthread_mutex_unlock(&mu_);
        return n;
      }
      std::function<void()> f = std::move(work_.front());
      work_.pop_front();
      pthread_mutex_unlock(&mu_);
      f();
      n++;
    }
  }
  void stop() {
    pthread_mutex_lock(&mu_);
    stopped_ = true;
    pthread_mutex_unlock(&mu_);
  }
  void reset() {
    pthread_mutex_lock(&mu_);
    stopped_ = false;
    pthread_mutex_unlock(&mu_);
  }

 private:
  pthread_mutex_t mu_;
  pthread_cond_t cv_;
  std::deque<std::function<void()>> work_;
  bool stopped_;
};

class socket_base {
 public:
  class receive_buffer_size {
   public:
    explicit receive_buffer_size(int v) : v_(v) {}
    int level() const { return SOL_SOCKET; }
    int name() const { return SO_RCVBUF; }
    const int *data() const { return &v_; }

   private:
    int v_;
  };
  class reuse_address {
   public:
    explicit reuse_address(bool v) : v_(v ? 1 : 0) {}
    int level() const { return SOL_SOCKET; }
    int name() const { return SO_REUSEADDR; }
    const int *data() const { return &v_; }

   private:
    int v_;
  };
};

namespace placeholders {
static const decltype(std::placeholders::_1) &error = std::placeholders::_1;
}  // namespace placeholders

namespace ip {

class address {
 public:
  address() : a_(htonl(INADDR_ANY)) {}
  static address from_string(const std::string &s) {
    address r;
    if (inet_pton(AF_INET, s.c_str(), &r.a_) != 1) throw boost::system::system_error(boost::system::error_code(EINVAL), "address " + s);
    return r;
  }
  uint32_t raw() const { return a_; }
  std::string to_string() const {
    char b[INET_ADDRSTRLEN];
    inet_ntop(AF_INET, &a_, b, sizeof(b));
    return b;
  }

 private:
  uint32_t a_;  // network order
};

class tcp {
 public:
  static tcp v4() { return tcp(); }

  class endpoint {
   public:
    endpoint() { memset(&sa_, 0, sizeof(sa_)); sa_.sin_family = AF_INET; }
    endpoint(const tcp &, unsigned short port) : endpoint() {
      sa_.sin_addr.s_addr = htonl(INADDR_ANY);
      sa_.sin_port = htons(port);
    }
    endpoint(const address &a, unsigned short port) : endpoint() {
      sa_.sin_addr.s_addr = a.raw();
      sa_.sin_port = htons(port);
    }
    const sockaddr *data() const { return reinterpret_cast<const sockaddr *>(&sa_); }
    socklen_t size() const { return sizeof(sa_); }
    unsigned short port() const { return ntohs(sa_.sin_port); }

   private:
    sockaddr_in sa_;
  };

  class socket {
   public:
    explicit socket(io_service &ios) : ios_(&ios), fd_(-1) {}
    ~socket() { close(); }
    socket(const socket &) = delete;
    socket &operator=(const socket &) = delete;

    void connect(const endpoint &ep) {
      boost::system::error_code ec;
      connect(ep, ec);
      if (ec) throw boost::system::system_error(ec, "connect");
    }
    void connect(const endpoint &ep, boost::system::error_code &ec) {
      close();
      fd_ = ::socket(AF_INET, SOCK_STREAM, 0);
      if (fd_ < 0 || ::connect(fd_, ep.data(), ep.size()) != 0) {
        ec = boost::system::error_code(errno);
        close();
        return;
      }
      nodelay();
      ec = boost::system::error_code();
    }
    void close() {
      if (fd_ >= 0) ::close(fd_);
      fd_ = -1;
    }
    bool is_open() const { return fd_ >= 0; }
    template <class Option>
    void set_option(const Option &o) {
      if (fd_ >= 0) setsockopt(fd_, o.level(), o.name(), o.data(), sizeof(*o.data()));
    }
    std::size_t send(const const_buffer &b) {
      const ssize_t r = ::send(fd_, b.data, b.size, MSG_NOSIGNAL);
      if (r < 0) throw boost::system::system_error(boost::system::error_code(errno), "send");
      return (std::size_t)r;
    }
    std::size_t receive(const mutable_buffer &b) {
      const ssize_t r = ::recv(fd_, b.data, b.size, 0);
      if (r < 0) throw boost::system::system_error(boost::system::error_code(errno), "receive");
      return (std::size_t)r;
    }
    io_service &get_io_service() { return *ios_; }
    int native_handle() const { return fd_; }
    int native() const { return fd_; }  // the older name of native_handle()
    void assign_accepted(int fd) {
      close();
      fd_ = fd;
      nodelay();
    }

   private:
    void nodelay() {
      int one = 1;
      setsockopt(fd_, IPPROTO_TCP, TCP_NODELAY, &one, sizeof(one));
    }
    io_service *ios_;
    int fd_;
  };

  class acceptor {
   public:
    typedef socket_base::reuse_address reuse_address;
    acceptor(io_service &ios, const endpoint &ep) : ios_(&ios), fd_(::socket(AF_INET, SOCK_STREAM, 0)) {
      if (fd_ < 0) throw boost::system::system_error(boost::system::error_code(errno), "socket");
      int one = 1;
      setsockopt(fd_, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
      if (::bind(fd_, ep.data(), ep.size()) != 0 || ::listen(fd_, 64) != 0) {
        const int e = errno;
        ::close(fd_);
        throw boost::system::system_error(boost::system::error_code(e), "bind/listen");
      }
    }
    ~acceptor() {
      if (fd_ >= 0) ::close(fd_);
    }
    template <class Option>
    void set_option(const Option &o) {
      setsockopt(fd_, o.level(), o.name(), o.data(), sizeof(*o.data()));
    }
    void listen(int backlog = 64) { ::listen(fd_, backlog); }  // already listening since construction
    void accept(socket &s) {
      int c;
      do {
        c = ::accept(fd_, nullptr, nullptr);
      } while (c < 0 && errno == EINTR);
      if (c < 0) throw boost::system::system_error(boost::system::error_code(errno), "accept");
      s.assign_accepted(c);
    }
    // Queues the accept on the io_service: run() performs it (blocking) and then calls
    // handler(error_code).
    template <class Handler>
    void async_accept(socket &s, Handler handler) {
      socket *sp = &s;
      int fd = fd_;
      ios_->post([sp, fd, handler]() mutable {
        int c;
        do {
          c = ::accept(fd, nullptr, nullptr);
        } while (c < 0 && errno == EINTR);
        boost::system::error_code ec;
        if (c < 0)
          ec = boost::system::error_code(errno);
        else
          sp->assign_accepted(c);
        handler(ec);
      });
    }
    io_service &get_io_service() { return *ios_; }

   private:
    io_service *ios_;
    int fd_;
  };
};

}  // namespace ip

// Reads exactly the buffer's size (blocking); throws on an error or a closed peer.
inline std::size_t read(ip::tcp::socket &s, const mutable_buffer &b) {
  std::size_t got = 0;
  while (got < b.size) {
    const ssize_t r = ::recv(s.native_handle(), (char *)b.data + got, b.size - got, 0);
    if (r < 0 && errno == EINTR) continue;
    if (r < 0) throw boost::system::system_error(boost::system::error_code(errno), "read");
    if (r == 0) throw boost::system::system_error(boost::system::error_code(ECONNRESET), "read: end of stream");
    got += (std::size_t)r;
  }
  return got;
}

// Writes the whole buffer (blocking); throws on an error.
inline std::size_t write(ip::tcp::socket &s, const const_buffer &b) {
  std::size_t sent = 0;
  while (sent < b.size) {
    const ssize_t r = ::send(s.native_handle(), (const char *)b.data + sent, b.size - sent, MSG_NOSIGNAL);
    if (r < 0 && errno == EINTR) continue;
    if (r < 0) throw boost::system::system_error(boost::system::error_code(errno), "write");
    sent += (std::size_t)r;
  }
  return sent;
}
inline std::size_t write(ip::tcp::socket &s, const mutable_buffer &b) { return write(s, const_buffer(b)); }

// Registers for the signals; the handlers are not called here: the signals keep their
// default action (a server stopped with SIGINT or SIGTERM ends its process).
class signal_set {
 public:
  signal_set(io_service &ios, int, int = 0, int = 0) : ios_(&ios) {}
  template <class Handler>
  void async_wait(Handler) {}

 private:
  io_service *ios_;
};

}  // namespace asio
}  // namespace boost

#endif
