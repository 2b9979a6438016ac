// Project-written stand-in: boost::begin (see iterator_range.hpp).  Test infrastructure only.
#include <boost/range/iterator_range.hpp>
