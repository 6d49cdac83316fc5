/* Stand-in for src/nemo/Simulation.hpp: the simulation interface. */
#ifndef NEMO_SIMULATION_HPP
#define NEMO_SIMULATION_HPP
#include <vector>
#include <utility>
#include <cstddef>
#include <nemo/config.h>
#include <nemo/types.h>
#include <nemo/ReadableNetwork.hpp>
namespace nemo {
class NEMO_BASE_DLL_PUBLIC Simulation : public ReadableNetwork
{
	public :
		virtual ~Simulation() { }
		typedef std::vector<unsigned> firing_output;
		typedef std::vector<unsigned> firing_stimulus;
		typedef std::vector< std::pair<unsigned, float> > current_stimulus;
		virtual const firing_output& step() = 0;
		virtual const firing_output& step(const firing_stimulus& fstim) = 0;
		virtual const firing_output& step(const current_stimulus& istim) = 0;
		virtual const firing_output& step(const firing_stimulus& fstim, const current_stimulus& istim) = 0;
		virtual void setNeuron(unsigned idx, unsigned nargs, const float args[]) = 0;
		virtual void setNeuronState(unsigned neuron, unsigned var, float value) = 0;
		virtual void setNeuronParameter(unsigned neuron, unsigned parameter, float value) = 0;
		virtual void applyStdp(float reward) = 0;
		virtual float getNeuronState(unsigned neuron, unsigned var) const = 0;
		virtual float getNeuronParameter(unsigned neuron, unsigned parameter) const = 0;
		virtual float getMembranePotential(unsigned neuron) const = 0;
		virtual const std::vector<synapse_id>& getSynapsesFrom(unsigned neuron) = 0;
		virtual unsigned long elapsedWallclock() const = 0;
		virtual unsigned long elapsedSimulation() const = 0;
		virtual void resetTimer() = 0;
	protected :
		Simulation() { }
	private :
		Simulation(const Simulation&);
		Simulation& operator=(const Simulation&);
};
}
#endif
