// Core value types of the TMFQS API (mirrors include/tmfqs/core/types.h of
// the reference: qubit 0 is the most significant bit of a state index; the
// amplitude buffer is interleaved [re0, im0, re1, im1, ...]).
#ifndef TMFQS_HOST_CORE_TYPES_H
#define TMFQS_HOST_CORE_TYPES_H

#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <utility>
#include <vector>

namespace tmfqs {

using QubitIndex = unsigned int;
using StateIndex = std::uint64_t;

struct Amplitude {
	double real;
	double imag;
};

using AmplitudesVector = std::vector<double>;

// Ordered list of values with the small vector-like surface the API uses.
template <typename T>
class IndexList {
	public:
		IndexList() = default;
		IndexList(std::initializer_list<T> init) : values_(init) {}
		explicit IndexList(std::vector<T> values) : values_(std::move(values)) {}
		size_t size() const noexcept { return values_.size(); }
		bool empty() const noexcept { return values_.empty(); }
		void reserve(size_t n) { values_.reserve(n); }
		void push_back(T v) { values_.push_back(v); }
		T operator[](size_t i) const { return values_[i]; }
		T &operator[](size_t i) { return values_[i]; }
		typename std::vector<T>::const_iterator begin() const noexcept { return values_.begin(); }
		typename std::vector<T>::const_iterator end() const noexcept { return values_.end(); }
		typename std::vector<T>::iterator begin() noexcept { return values_.begin(); }
		typename std::vector<T>::iterator end() noexcept { return values_.end(); }
		const std::vector<T> &values() const noexcept { return values_; }

	private:
		std::vector<T> values_;
};

using QubitList = IndexList<QubitIndex>;
using BasisStateList = IndexList<StateIndex>;

}  // namespace tmfqs

#endif
