// Page codec for the contest's 8 KiB column pages (header-only, host side).
//
// Writers follow the packing rule of the contest's row->page converter
// (src/build_table.cpp:456-660 of the contest repository): a non-null fixed-width
// value is added while  begin + (values+1)*width + (rows/8 + 1) <= 8192,  a null
// while  begin + values*width + (rows/8 + 1) <= 8192;  for strings the offsets
// (2 B each) and bytes take the place of the values, and a string longer than
// PAGE_SIZE - 7 gets its own run of long-string pages (0xffff then 0xfffe).
// Any packing that satisfies the format is valid input to the engine; these
// rules only make pages full.
//
// Pages are obtained from a caller-supplied allocator so that the same writer
// fills `Column`s (new Page) or one contiguous buffer (generators).
#pragma once

#include "plan.h"

#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace contest_pages {

using PageAlloc = std::function<Page*()>;

inline uint16_t rd16(const std::byte* p) {
    uint16_t v;
    std::memcpy(&v, p, 2);
    return v;
}
inline void wr16(std::byte* p, uint16_t v) { std::memcpy(p, &v, 2); }

// Byte offset of the first value in a fixed-width page.
constexpr size_t value_begin(size_t width) { return width == 8 ? 8 : 4; }

// Rows a page of this fixed width holds when no row is null.
constexpr size_t full_page_rows(size_t width) {
    size_t n = 0;
    while (value_begin(width) + (n + 1) * width + (n / 8 + 1) <= PAGE_SIZE) n++;
    return n;
}

// Writer for INT32 (width 4), INT64 / FP64 (width 8) columns.
class FixedWriter {
    public:
    FixedWriter(size_t width, PageAlloc alloc) : width_(width), alloc_(std::move(alloc)) {
        bitmap_.assign(PAGE_SIZE, 0);
        values_.resize(PAGE_SIZE);
    }
    void append(const void* value) {
        if (value_begin(width_) + (nvalues_ + 1) * width_ + (nrows_ / 8 + 1) > PAGE_SIZE) flush();
        std::memcpy(values_.data() + nvalues_ * width_, value, width_);
        bitmap_[nrows_ / 8] |= uint8_t(1u << (nrows_ % 8));
        nvalues_++;
        nrows_++;
    }
    void append_null() {
        if (value_begin(width_) + nvalues_ * width_ + (nrows_ / 8 + 1) > PAGE_SIZE) flush();
        nrows_++;
    }
    void finish() {
        if (nrows_) flush();
    }

    private:
    void flush() {
        Page* page = alloc_();
        std::byte* p = page->data;
        std::memset(p, 0, PAGE_SIZE);
        wr16(p, uint16_t(nrows_));
        wr16(p + 2, uint16_t(nvalues_));
        std::memcpy(p + value_begin(width_), values_.data(), nvalues_ * width_);
        size_t nb = (nrows_ + 7) / 8;
        std::memcpy(p + PAGE_SIZE - nb, bitmap_.data(), nb);
        std::memset(bitmap_.data(), 0, nb);
        nrows_ = nvalues_ = 0;
    }
    size_t width_;
    PageAlloc alloc_;
    std::vector<uint8_t> bitmap_;
    std::vector<uint8_t> values_;
    size_t nrows_ = 0, nvalues_ = 0;
};

// Writer for VARCHAR columns.
class StringWriter {
    public:
    explicit StringWriter(PageAlloc alloc) : alloc_(std::move(alloc)) {
        bitmap_.assign(PAGE_SIZE, 0);
    }
    static constexpr size_t kMaxShort = PAGE_SIZE - 7;

    void append(std::string_view s) {
        if (s.size() > kMaxShort) {
            if (nrows_) flush();
            size_t off = 0;
            bool first = true;
            while (off < s.size()) {
                size_t n = std::min(s.size() - off, PAGE_SIZE - 4);
                Page* page = alloc_();
                std::byte* p = page->data;
                std::memset(p, 0, PAGE_SIZE);
                wr16(p, first ? 0xffff : 0xfffe);
                wr16(p + 2, uint16_t(n));
                std::memcpy(p + 4, s.data() + off, n);
                off += n;
                first = false;
            }
            return;
        }
        if (4 + (offsets_.size() + 1) * 2 + chars_.size() + s.size() + (nrows_ / 8 + 1) > PAGE_SIZE) flush();
        chars_.insert(chars_.end(), s.begin(), s.end());
        offsets_.push_back(uint16_t(chars_.size()));
        bitmap_[nrows_ / 8] |= uint8_t(1u << (nrows_ % 8));
        nrows_++;
    }
    void append_null() {
        if (4 + offsets_.size() * 2 + chars_.size() + (nrows_ / 8 + 1) > PAGE_SIZE) flush();
        nrows_++;
    }
    void finish() {
        if (nrows_) flush();
    }

    private:
    void flush() {
        Page* page = alloc_();
        std::byte* p = page->data;
        std::memset(p, 0, PAGE_SIZE);
        wr16(p, uint16_t(nrows_));
        wr16(p + 2, uint16_t(offsets_.size()));
        std::memcpy(p + 4, offsets_.data(), offsets_.size() * 2);
        std::memcpy(p + 4 + offsets_.size() * 2, chars_.data(), chars_.size());
        size_t nb = (nrows_ + 7) / 8;
        std::memcpy(p + PAGE_SIZE - nb, bitmap_.data(), nb);
        std::memset(bitmap_.data(), 0, nb);
        nrows_ = 0;
        offsets_.clear();
        chars_.clear();
    }
    PageAlloc alloc_;
    std::vector<uint8_t> bitmap_;
    std::vector<uint16_t> offsets_;
    std::vector<char> chars_;
    size_t nrows_ = 0;
};

// One decoded cell. `kind` is the column's DataType or -1 for NULL.
struct Cell {
    int kind = -1;
    uint64_t bits = 0;  // INT32 sign-extended to 64 bits, INT64, or FP64 bit pattern
    std::string str;    // VARCHAR
};

// Calls fn(row_index, const Cell&) for every row of a column, in row order.
template <typename Fn>
void decode_column(DataType type, const Page* const* pages, size_t num_pages, Fn&& fn) {
    size_t row = 0;
    Cell cell;
    for (size_t pi = 0; pi < num_pages; pi++) {
        const std::byte* p = pages[pi]->data;
        uint16_t nrows = rd16(p);
        if (type == DataType::VARCHAR && nrows == 0xffff) {
            cell.kind = int(DataType::VARCHAR);
            cell.str.assign(reinterpret_cast<const char*>(p + 4), rd16(p + 2));
            while (pi + 1 < num_pages && rd16(pages[pi + 1]->data) == 0xfffe) {
                pi++;
                const std::byte* q = pages[pi]->data;
                cell.str.append(reinterpret_cast<const char*>(q + 4), rd16(q + 2));
            }
            fn(row++, cell);
            continue;
        }
        if (type == DataType::VARCHAR && nrows == 0xfffe)
            throw std::runtime_error("long-string continuation page without a start page");
        const uint8_t* bitmap = reinterpret_cast<const uint8_t*>(p + PAGE_SIZE - (nrows + 7) / 8);
        size_t dense = 0;
        uint16_t nvalues = rd16(p + 2);
        const char* chars = reinterpret_cast<const char*>(p + 4 + 2 * size_t(nvalues));
        for (size_t i = 0; i < nrows; i++) {
            bool valid = (bitmap[i / 8] >> (i % 8)) & 1;
            if (!valid) {
                cell.kind = -1;
                fn(row++, cell);
                continue;
            }
            cell.kind = int(type);
            switch (type) {
            case DataType::INT32: {
                int32_t v;
                std::memcpy(&v, p + 4 + 4 * dense, 4);
                cell.bits = uint64_t(int64_t(v));
                break;
            }
            case DataType::INT64:
            case DataType::FP64:
                std::memcpy(&cell.bits, p + 8 + 8 * dense, 8);
                break;
            case DataType::VARCHAR: {
                uint16_t end = rd16(p + 4 + 2 * dense);
                uint16_t begin = dense ? rd16(p + 4 + 2 * (dense - 1)) : 0;
                cell.str.assign(chars + begin, chars + end);
                break;
            }
            }
            dense++;
            fn(row++, cell);
        }
    }
}

// Rows stored in a column's pages (long-string continuation pages hold none).
inline size_t count_rows(DataType type, const Page* const* pages, size_t num_pages) {
    size_t n = 0;
    for (size_t i = 0; i < num_pages; i++) {
        uint16_t r = rd16(pages[i]->data);
        if (type == DataType::VARCHAR && r >= 0xfffe)
            n += (r == 0xffff);
        else
            n += r;
    }
    return n;
}

} // namespace contest_pages
