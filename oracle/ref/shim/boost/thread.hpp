/* Test-infrastructure shim: the few boost::thread names the reference's scene and
 * scheduler headers use, backed by std::thread.  The oracle never starts the
 * reference's scheduler. */
#pragma once
#include <thread>
#include <mutex>
#include <functional>
#include <vector>
namespace boost {
class thread {
public:
    thread() {}
    template <class F, class... A> explicit thread(F &&f, A &&...a)
        : t_(std::forward<F>(f), std::forward<A>(a)...) {}
    void join() { if (t_.joinable()) t_.join(); }
    void interrupt() {}
    bool joinable() const { return t_.joinable(); }
private:
    std::thread t_;
};
class mutex : public std::mutex {
public:
    typedef std::unique_lock<std::mutex> scoped_lock;
};
using std::bind;
class thread_group {
public:
    ~thread_group() { for (auto *t : ts_) { t->join(); delete t; } }
    template <class F> thread *create_thread(F f) { ts_.push_back(new thread(f)); return ts_.back(); }
    void add_thread(thread *t) { ts_.push_back(t); }
    void join_all() { for (auto *t : ts_) t->join(); }
    std::size_t size() const { return ts_.size(); }
    void interrupt_all() {}
private:
    std::vector<thread *> ts_;
};
namespace this_thread { template <class T> void sleep(const T &) {} inline void yield() {} }
namespace posix_time { struct milliseconds { explicit milliseconds(long) {} };
struct microseconds { explicit microseconds(long) {} }; }
}
