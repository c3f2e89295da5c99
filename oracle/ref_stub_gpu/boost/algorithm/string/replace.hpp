#include "../../../../ref_stub/boost/algorithm/string/replace.hpp"
