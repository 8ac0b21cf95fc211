#pragma once
#include <mutex>
namespace boost { using std::recursive_mutex; }
