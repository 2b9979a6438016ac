// Project-written stand-in: boost::size (see iterator_range.hpp).
#include <boost/range/iterator_range.hpp>
