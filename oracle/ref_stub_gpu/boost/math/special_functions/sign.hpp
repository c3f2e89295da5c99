#include "../../../../ref_stub/boost/math/special_functions/sign.hpp"
