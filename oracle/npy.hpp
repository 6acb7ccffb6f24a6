#pragma once
// ORACLE (test infrastructure only): minimal .npy writer for fixture dumps.
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace apf_oracle
{
    template<class T> inline const char* npy_descr();
    template<> inline const char* npy_descr<double>() { return "<f8"; }
    template<> inline const char* npy_descr<float>() { return "<f4"; }
    template<> inline const char* npy_descr<int>() { return "<i4"; }
    template<> inline const char* npy_descr<long long>() { return "<i8"; }
    template<> inline const char* npy_descr<std::int64_t>() { return "<i8"; }

    template<class T>
    inline void write_npy(const std::string& path, const T* data, std::vector<std::size_t> shape)
    {
        std::string sh = "(";
        std::size_t count = 1;
        for (std::size_t i = 0; i < shape.size(); ++i)
        {
            sh += std::to_string(shape[i]);
            sh += (shape.size() == 1 || i + 1 < shape.size()) ? "," : "";
            if (i + 1 < shape.size()) sh += " ";
            count *= shape[i];
        }
        sh += ")";
        std::string header = std::string("{'descr': '") + npy_descr<T>() + "', 'fortran_order': False, 'shape': " + sh + ", }";
        const std::size_t total = 10 + header.size() + 1;
        header.append((64 - total % 64) % 64, ' ');
        header.push_back('\n');
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) throw std::runtime_error("cannot open " + path);
        const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
        std::fwrite(magic, 1, 8, f);
        const std::uint16_t hl = static_cast<std::uint16_t>(header.size());
        std::fwrite(&hl, 2, 1, f);
        std::fwrite(header.data(), 1, header.size(), f);
        if (count) std::fwrite(data, sizeof(T), count, f);
        std::fclose(f);
    }

    template<class T>
    inline void write_npy(const std::string& path, const std::vector<T>& v)
    {
        write_npy(path, v.data(), {v.size()});
    }
}
