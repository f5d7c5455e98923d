#pragma once

// Row-major dense matrices, owning (Matrix) and borrowed (MatrixView): the argument types of the
// reference's index API (include/vecdex/matrix.hpp:22-137), kept so callers switch without
// changing their code.

#include <cassert>
#include <cstddef>
#include <functional>
#include <limits>
#include <span>
#include <stdexcept>
#include <vector>

namespace vdx {

template <typename T>
class Matrix {
public:
    explicit Matrix(std::size_t dim) : Matrix(0, dim) {}

    Matrix(std::size_t rows, std::size_t dim) : dim_(dim) {
        if (dim == 0) {
            throw std::invalid_argument("Matrix: dim must be positive");
        }
        if (rows > std::numeric_limits<std::size_t>::max() / dim) {
            throw std::length_error("Matrix: rows * dim overflows size_t");
        }
        data_.resize(rows * dim);
    }

    std::size_t rows() const noexcept { return data_.size() / dim_; }
    std::size_t dim() const noexcept { return dim_; }
    bool empty() const noexcept { return data_.empty(); }

    std::span<T> row(std::size_t i) noexcept {
        assert(i < rows());
        return {data_.data() + i * dim_, dim_};
    }
    std::span<const T> row(std::size_t i) const noexcept {
        assert(i < rows());
        return {data_.data() + i * dim_, dim_};
    }
    std::span<T> data() noexcept { return data_; }
    std::span<const T> data() const noexcept { return data_; }

    void reserve_rows(std::size_t rows) {
        if (rows > std::numeric_limits<std::size_t>::max() / dim_) {
            throw std::length_error("Matrix: rows * dim overflows size_t");
        }
        data_.reserve(rows * dim_);
    }

    // Appends values.size() / dim() rows. `values` may alias this matrix's own storage.
    void append(std::span<const T> values) {
        if (values.size() % dim_ != 0) {
            throw std::invalid_argument("Matrix::append: size is not a multiple of dim");
        }
        const T* begin = data_.data();
        const T* end = begin + data_.size();
        const bool aliases = !values.empty() && !std::less<const T*>{}(values.data(), begin) &&
                             std::less<const T*>{}(values.data(), end);
        if (aliases) {
            const auto offset = static_cast<std::size_t>(values.data() - begin);
            const std::size_t old = data_.size();
            data_.resize(old + values.size());
            for (std::size_t i = 0; i < values.size(); ++i) {
                data_[old + i] = data_[offset + i];
            }
        } else {
            data_.insert(data_.end(), values.begin(), values.end());
        }
    }

private:
    std::size_t dim_;
    std::vector<T> data_;
};

template <typename T>
class MatrixView {
public:
    MatrixView(std::span<const T> data, std::size_t dim) : data_(data), dim_(dim) {
        if (dim == 0) {
            throw std::invalid_argument("MatrixView: dim must be positive");
        }
        if (data.size() % dim != 0) {
            throw std::invalid_argument("MatrixView: size is not a multiple of dim");
        }
    }
    MatrixView(const Matrix<T>& m) noexcept  // NOLINT(*-explicit-constructor): as std::span
        : data_(m.data()), dim_(m.dim()) {}

    std::size_t rows() const noexcept { return data_.size() / dim_; }
    std::size_t dim() const noexcept { return dim_; }
    bool empty() const noexcept { return data_.empty(); }
    std::span<const T> row(std::size_t i) const noexcept {
        assert(i < rows());
        return data_.subspan(i * dim_, dim_);
    }
    std::span<const T> data() const noexcept { return data_; }

private:
    std::span<const T> data_;
    std::size_t dim_;
};

}  // namespace vdx
