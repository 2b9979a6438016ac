// Project-written stand-in (see variant.hpp).
#include <boost/variant/variant.hpp>
