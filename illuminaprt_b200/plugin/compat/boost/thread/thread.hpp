#pragma once
#include <thread>
namespace boost { struct thread : std::thread { using std::thread::thread; static unsigned hardware_concurrency() { return std::thread::hardware_concurrency(); } }; }
