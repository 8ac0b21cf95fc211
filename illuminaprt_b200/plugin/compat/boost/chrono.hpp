#pragma once
#include <chrono>
namespace boost { namespace chrono = std::chrono; }
