/* Test-infrastructure shim: the reference's log timestamps only need a printable
 * time.  No Boost is installed; this replaces ptime/microsec_clock with a stub. */
#pragma once
#include <string>
namespace boost { namespace posix_time {
struct ptime { template <class T> explicit ptime(T) {} };
struct microsec_clock { static int local_time() { return 0; } };
inline std::string to_simple_string(const ptime &) { return "0"; }
} }
