#include <boost/config.hpp>
