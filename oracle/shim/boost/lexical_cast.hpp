// Minimal stand-in for boost::lexical_cast<std::string>(x) (project-written).
#pragma once
#include <sstream>
#include <string>
namespace boost {
template <class T, class S> T lexical_cast(const S& v) { std::ostringstream o; o << v; return o.str(); }
}
