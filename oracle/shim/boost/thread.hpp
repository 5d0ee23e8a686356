/*
 * Stand-in for boost::thread over std::thread.  ORACLE INFRASTRUCTURE ONLY:
 * lets the reference's fusion sources compile into oracle/_ref/.
 */
#ifndef FF_ORACLE_SHIM_BOOST_THREAD_HPP
#define FF_ORACLE_SHIM_BOOST_THREAD_HPP
#include <thread>
#include <utility>
namespace boost {
class thread {
 public:
  template <typename F, typename... A>
  explicit thread(F f, A... a) : t_(f, a...) {}
  void join() {
    if (t_.joinable()) t_.join();
  }
  ~thread() {
    if (t_.joinable()) t_.join();
  }

 private:
  std::thread t_;
};
}  // namespace boost
#endif
