#pragma once
#include <string>
#include <cstddef>
// File mapping is only used by the reference's persistent mesh, which the
// nothing built here uses; these types exist so its headers compile.
namespace boost { namespace iostreams {
struct mapped_file_source { bool is_open() const { return false; } const char *data() const { return 0; } std::size_t size() const { return 0; } void close() {} void open(const std::string &) {} };
struct mapped_file { enum mapmode { readonly, readwrite, priv }; bool is_open() const { return false; } char *data() const { return 0; } const char *const_data() const { return 0; } std::size_t size() const { return 0; } void close() {} template <class... A> void open(const A &...) {} };
struct mapped_file_params { std::string path; mapped_file::mapmode flags; std::size_t new_file_size = 0; };
} }
