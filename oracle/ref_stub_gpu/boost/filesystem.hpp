#include "../../ref_stub/boost/filesystem.hpp"
