// dt/details/status.hpp -- C ABI status codes to C++ exceptions, and the per-device default context used by
// the free functions of namespace dt.
//
// The reference reports CUDA failures as std::runtime_error after the call
// (dt/src/generalised_distance_transform.cu:136-137, dt/src/transfert.cpp:16-17) and allocation failure by
// throwing (dt/include/dt/details/image2d_data_gpu.hpp:29-30).  Here every non-OK status of the C ABI throws
// dt::error, a std::runtime_error carrying the status and the library's message.
#pragma once

#include <cstdlib>
#include <stdexcept>
#include <string>

#include "dtb.h"

namespace dt
{
  class error : public std::runtime_error
  {
  public:
    error(dtb_status status, const std::string& what) : std::runtime_error(what), m_status(status) {}
    dtb_status status() const noexcept { return m_status; }

  private:
    dtb_status m_status;
  };

  namespace details
  {
    inline void check(dtb_status s, const char* what, dtb_context ctx = nullptr)
    {
      if (s == DTB_OK)
        return;
      std::string msg = std::string(what) + ": " + dtb_status_string(s);
      if (ctx)
      {
        const char* m = dtb_context_message(ctx);
        if (m && *m)
          msg += std::string(" (") + m + ")";
      }
      throw error(s, msg);
    }

    // Device the free functions run on: DT_DEVICE from the environment, else 0 (the reference runs on device 0,
    // dt/src/generalised_distance_transform_task.cu:186).
    inline int default_device()
    {
      const char* e = std::getenv("DT_DEVICE");
      return e ? std::atoi(e) : 0;
    }

    // One library context per process for the free functions, created on first use and released at exit.
    // Calls through it are serialised by the library (a context is used by one call at a time).  The context
    // is created inside the holder's constructor, so the CUDA runtime is initialised before the holder's
    // destructor is registered and that destructor runs before the runtime shuts down.
    inline dtb_context context()
    {
      struct holder
      {
        dtb_context ctx    = nullptr;
        dtb_status  status = DTB_OK;
        holder() { status = dtb_context_create(default_device(), &ctx); }
        ~holder()
        {
          if (ctx)
            dtb_context_destroy(ctx);
        }
      };
      static holder h;
      check(h.status, "dtb_context_create");
      return h.ctx;
    }
  } // namespace details
} // namespace dt
