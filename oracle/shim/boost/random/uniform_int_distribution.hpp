// Stand-in for boost::random::uniform_int_distribution<> (project-written).
#pragma once
#include <random>
namespace boost { namespace random { template <class T = int> using uniform_int_distribution = std::uniform_int_distribution<T>; } }
