/* Minimal stand-in for boost::filesystem over std::filesystem (directory creation only). */
#pragma once
#include <filesystem>
#include <system_error>
namespace boost { namespace filesystem = std::filesystem; namespace system { typedef std::error_code error_code; } }
