/* Build stand-in for Boost, which this image lacks: boost::any mapped onto std::any. */
#pragma once
#include <any>
namespace boost {
using any = std::any;
template <class T> T any_cast(any &a) { return std::any_cast<T>(a); }
template <class T> T any_cast(const any &a) { return std::any_cast<T>(a); }
}
