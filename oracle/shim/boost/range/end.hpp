// Project-written stand-in: boost::end (see iterator_range.hpp).  Test infrastructure only.
#include <boost/range/iterator_range.hpp>
