// Stand-in for boost::typeindex, used only to compile the reference's own
// scalar operators as a test oracle (the operators never call it).
#pragma once
#include <typeindex>
#include <typeinfo>
#ifndef BOOST_NOEXCEPT
#define BOOST_NOEXCEPT noexcept
#endif
namespace boost {
namespace typeindex {
typedef std::type_index type_index;
template <typename T>
inline type_index type_id() { return std::type_index(typeid(T)); }
}  // namespace typeindex
}  // namespace boost
