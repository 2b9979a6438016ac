// Project-written stand-in (see variant/variant.hpp).
#include <boost/variant/variant.hpp>
