// Stand-in: boost::recursive_mutex is provided by the boost/thread.hpp shim.
#include <boost/thread.hpp>
