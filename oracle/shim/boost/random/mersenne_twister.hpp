// Stand-in: the reference only names boost::random::mt19937 (project-written).
#pragma once
#include <random>
namespace boost { namespace random { using std::mt19937; } }
