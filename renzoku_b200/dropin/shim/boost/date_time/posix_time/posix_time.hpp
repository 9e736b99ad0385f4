/* Build stand-in for Boost, which this image lacks: the reference's log timestamps only
 * need a printable time, so ptime / microsec_clock are stubs. */
#pragma once
#include <string>
namespace boost { namespace posix_time {
struct ptime { template <class T> explicit ptime(T) {} };
struct microsec_clock { static int local_time() { return 0; } };
inline std::string to_simple_string(const ptime &) { return "0"; }
} }
