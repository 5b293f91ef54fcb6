// dt/random_image2d.hpp -- CPU image of uniformly random integer pixels over the full range of T, reference
// dt::random_image2d (dt/include/dt/random_image2d.hpp:9-24; seeded from std::random_device as there).
#pragma once

#include <dt/image2d.hpp>

#include <cstdint>
#include <limits>
#include <random>

namespace dt
{
  template <typename T>
  image2d<T> random_image2d(int width, int height)
  {
    std::random_device                  rd;
    std::mt19937_64                     gen(rd());
    std::uniform_int_distribution<long long> pick(static_cast<long long>(std::numeric_limits<T>::min()),
                                                  static_cast<long long>(std::numeric_limits<T>::max()));
    image2d<T> img(width, height);
    for (int y = 0; y < height; ++y)
      for (int x = 0; x < width; ++x)
        img(x, y) = static_cast<T>(pick(gen));
    return img;
  }
} // namespace dt
