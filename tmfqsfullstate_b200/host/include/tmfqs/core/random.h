// Random sources for measurement (include/tmfqs/core/random.h:15-58).
#ifndef TMFQS_HOST_CORE_RANDOM_H
#define TMFQS_HOST_CORE_RANDOM_H

#include <cstdint>
#include <random>

namespace tmfqs {

class IRandomSource {
	public:
		virtual ~IRandomSource() = default;
		// A value in [0, 1).
		virtual double nextUnitDouble() = 0;
};

// std::mt19937 + uniform_real_distribution<double>(0, 1): the stream the
// reference's measure() consumes.
class Mt19937RandomSource : public IRandomSource {
	public:
		Mt19937RandomSource();  // seeded from std::random_device
		explicit Mt19937RandomSource(uint32_t seed);
		double nextUnitDouble() override;
		void reseed(uint32_t seed);

	private:
		std::mt19937 engine_;
		std::uniform_real_distribution<double> distribution_{0.0, 1.0};
};

}  // namespace tmfqs

#endif
