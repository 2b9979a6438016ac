// Project-written stand-in: boost::begin (see iterator_range.hpp).  Used to build the reference's code in this image, which has no Boost.
#include <boost/range/iterator_range.hpp>
