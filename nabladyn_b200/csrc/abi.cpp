// The error channel and version of the C-ABI.

#include <string>

#include "nabladyn_b200.h"

namespace nd {

namespace {
thread_local std::string message;
}

void set_error(const std::string& text)
{
    message = text;
}

const char* last_error()
{
    return message.c_str();
}

}  // namespace nd

extern "C" const char* nd_last_error(void)
{
    return nd::last_error();
}

extern "C" int nd_abi_version(void)
{
    return 1;
}
