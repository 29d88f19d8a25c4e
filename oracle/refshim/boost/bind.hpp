// Stand-in for boost/bind.hpp: the reference binds member functions to an
// object pointer (or shared_ptr) and fixed arguments only.
#pragma once
#include <functional>
namespace boost {
using std::bind;
}
