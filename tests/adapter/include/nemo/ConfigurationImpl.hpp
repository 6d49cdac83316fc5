/* Stand-in for src/nemo/ConfigurationImpl.hpp: the configuration a
 * backend is created with.  The reference keeps the STDP function in a
 * boost::optional; std::optional offers the same operations. */
#ifndef NEMO_CONFIGURATION_IMPL_HPP
#define NEMO_CONFIGURATION_IMPL_HPP
#include <optional>
#include <string>
#include <nemo/config.h>
#include "StdpFunction.hpp"
#include "types.h"
namespace nemo {
class NEMO_BASE_DLL_PUBLIC ConfigurationImpl
{
	public:
		ConfigurationImpl() : m_writeOnlySynapses(false), m_fractionalBits(20), m_cudaPartitionSize(0),
			m_cudaDevice(0), m_backend(NEMO_BACKEND_CUDA) { }
		void setCudaPartitionSize(unsigned ps) { m_cudaPartitionSize = ps; }
		unsigned cudaPartitionSize() const { return m_cudaPartitionSize; }
		void setCudaDevice(unsigned device) { m_cudaDevice = device; }
		unsigned cudaDevice() const { return m_cudaDevice; }
		void setStdpFunction(const std::vector<float>& prefire, const std::vector<float>& postfire,
				float minE, float maxE, float minI, float maxI) {
			m_stdpFn.emplace(prefire, postfire, minE, maxE, minI, maxI);
		}
		const std::optional<StdpFunction>& stdpFunction() const { return m_stdpFn; }
		void setWriteOnlySynapses() { m_writeOnlySynapses = true; }
		bool writeOnlySynapses() const { return m_writeOnlySynapses; }
		void setFractionalBits(unsigned bits) { m_fractionalBits = (int) bits; }
		unsigned fractionalBits() const { return (unsigned) m_fractionalBits; }
		bool fractionalBitsSet() const { return m_fractionalBits != -1; }
		void setBackend(backend_t backend) { m_backend = backend; }
		backend_t backend() const { return m_backend; }
		void setBackendDescription(const char* descr) { m_backendDescription.assign(descr); }
		const char* backendDescription() const { return m_backendDescription.c_str(); }
	private:
		std::optional<StdpFunction> m_stdpFn;
		bool m_writeOnlySynapses;
		int m_fractionalBits;
		unsigned m_cudaPartitionSize;
		unsigned m_cudaDevice;
		backend_t m_backend;
		std::string m_backendDescription;
};
}
#endif
