/* Stand-in for src/nemo/StdpFunction.hpp: the STDP window and limits. */
#ifndef NEMO_STDP_FUNCTION
#define NEMO_STDP_FUNCTION
#include <vector>
#include <nemo/config.h>
#include <nemo/internal_types.h>
namespace nemo {
class NEMO_BASE_DLL_PUBLIC StdpFunction
{
	public :
		StdpFunction(const std::vector<float>& prefire, const std::vector<float>& postfire,
				float minExcitatoryWeight, float maxExcitatoryWeight,
				float minInhibitoryWeight, float maxInhibitoryWeight) :
			m_prefire(prefire), m_postfire(postfire),
			m_minExcitatoryWeight(minExcitatoryWeight), m_maxExcitatoryWeight(maxExcitatoryWeight),
			m_minInhibitoryWeight(minInhibitoryWeight), m_maxInhibitoryWeight(maxInhibitoryWeight) { }
		const std::vector<float>& prefire() const { return m_prefire; }
		const std::vector<float>& postfire() const { return m_postfire; }
		float minInhibitoryWeight() const { return m_minInhibitoryWeight; }
		float maxInhibitoryWeight() const { return m_maxInhibitoryWeight; }
		float minExcitatoryWeight() const { return m_minExcitatoryWeight; }
		float maxExcitatoryWeight() const { return m_maxExcitatoryWeight; }
	private :
		std::vector<float> m_prefire;
		std::vector<float> m_postfire;
		float m_minExcitatoryWeight;
		float m_maxExcitatoryWeight;
		float m_minInhibitoryWeight;
		float m_maxInhibitoryWeight;
};
}
#endif
