// Status codes and error text shared by the translation units of libfluidcuda.so. Every C entry
// point runs its body through guarded(): a Failure thrown by fail() becomes its status code,
// and the message is kept per thread for fc_last_error().
#pragma once

#include "../../include/fluidcuda.h"

#include <new>
#include <string>

namespace fc
{

extern thread_local std::string last_error;

struct Failure
{
    int status;
};

[[noreturn]] void fail(int status, const char* format, ...);

template <typename F> int guarded(F&& body)
{
    try
    {
        body();
        return FC_OK;
    }
    catch (const Failure& f)
    {
        return f.status;
    }
    catch (const std::bad_alloc&)
    {
        last_error = "host allocation failed";
        return FC_ERR_OUT_OF_MEMORY;
    }
    catch (...)
    {
        last_error = "unexpected exception";
        return FC_ERR_CUDA;
    }
}

} // namespace fc
