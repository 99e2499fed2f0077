// twisty_full_experiment -- drop-in for the reference's CLI driver Experiments/FullExperiment.cpp.
//
//   twisty_full_experiment config.json|config.yaml [--histogram]
//
// Reads the reference's experiment config (JSON, or the same keys in YAML), creates
// <experimentDir>/<name>/<timestamp>/ and copies the config there, runs the experiment on
// the B200 through the runner classes of include/twisty_b200_runner.hpp, and writes
// Results.dat with the lines the reference writes (FullExperiment.cpp:241-262), plus the
// log10 weight and the relative standard error.
#include "twisty_b200_runner.hpp"

#include <chrono>
#include <ctime>
#include <iomanip>
#include <iostream>

namespace {

std::string time_for_file_name()
{
    // GetCurrentTimeForFileName (Twisty/ExperimentRunner.cpp:30-38)
    const std::time_t t = std::time(nullptr);
    std::stringstream ss;
    ss << std::put_time(std::localtime(&t), "%F_%T");
    std::string s = ss.str();
    for (char &c : s)
        if (c == ':') c = '-';
    return s;
}

std::string format_duration(long long ms)
{
    // format_duration (Twisty/ExperimentRunner.cpp:14-28)
    const long long h = ms / 3600000, m = (ms / 60000) % 60, s = (ms / 1000) % 60, r = ms % 1000;
    std::stringstream ss;
    ss << h << " Hours : " << m << " Minutes : " << s << " Seconds : " << r << " Milliseconds";
    return ss.str();
}

}  // namespace

int main(int argc, char **argv)
{
    using namespace twisty::b200;
    if (argc < 2) {
        std::cout << "Call as: " << argv[0] << " configFilename" << std::endl;
        return 1;
    }
    // --histogram: also write histogram.txt (the reference's always-on path-weight histogram)
    const bool histogram = argc > 2 && std::string(argv[2]) == "--histogram";
    std::ifstream f(argv[1]);
    if (!f.is_open()) {
        std::cout << "Failed to open: " << argv[1] << std::endl;
        return 1;
    }
    std::stringstream buf;
    buf << f.rdbuf();
    const std::string path = argv[1];
    const bool yaml = path.size() > 5 && (path.rfind(".yaml") == path.size() - 5 || path.rfind(".yml") == path.size() - 4);
    BoundaryConditions bc;
    std::string err;
    ExperimentRunner::ExperimentParameters params =
          ExperimentRunner::ParseExperimentParamsFromConfig(buf.str(), yaml, &bc, &err);
    if (!err.empty()) {
        std::cout << "What: " << err << std::endl;
        return 1;
    }
    // experimentDir/name/timestamp/ (FullExperiment.cpp:35-39)
    {
        // the name and dir are not part of the C ABI params; read them from the config text
        auto grab = [&](const std::string &key) {
            const std::string t = buf.str();
            const size_t k = t.find("\"" + key + "\"");
            if (k == std::string::npos) return std::string();
            const size_t q1 = t.find('"', t.find(':', k) + 1), q2 = t.find('"', q1 + 1);
            return t.substr(q1 + 1, q2 - q1 - 1);
        };
        const std::string name = grab("name"), dir = grab("experimentDir");
        if (!name.empty()) params.experimentName = name;
        params.experimentDirPath = (dir.empty() ? std::string(".") : dir) + "/" + params.experimentName + "/" +
                                   time_for_file_name() + "/";
    }
    std::filesystem::create_directories(params.experimentDirPath);
    std::filesystem::copy_file(argv[1], params.experimentDirPath + "/" + params.experimentName + (yaml ? ".yaml" : ".json"),
                               std::filesystem::copy_options::overwrite_existing);
    params.perExperimentDirSubfolder = "main";
    params.outputHistogram = histogram;
    std::cout << "Experiment Path Count: " << params.numPathsInExperiment << std::endl;
    FullExperimentRunnerOptimalPerturbOptimized_GPU runner(params);
    std::optional<ExperimentRunner::ExperimentResults> results = runner.RunExperiment(bc);
    if (!results) {
        std::cout << "Experiment failed: no results returned. " << runner.lastError() << std::endl;
        return 1;
    }
    const auto &r = *results;
    const long double avg = r.experimentWeight / (long double)std::max<uint64_t>(r.totalPathsGenerated, 1);
    std::cout << "Paths Generated: " << r.totalPathsGenerated << std::endl;
    std::cout << "\tTotal experiment weight: " << r.experimentWeight << " (log10 " << std::setprecision(12)
              << r.experimentWeightLog10 << ")" << std::endl;
    std::cout << "\tAvg path weight: " << avg << std::endl;
    std::ofstream ofs(params.experimentDirPath + "/Results.dat");
    ofs << "Scatter value: " << params.weightingParameters.scatter << std::endl;
    ofs << "\tTotal experiment weight: " << r.experimentWeight << std::endl;
    ofs << "\tAvg path weight: " << avg << std::endl;
    ofs << "\tTotal experiment time (ms) " << format_duration(r.totalExperimentMs) << std::endl;
    ofs << "\tSetup time (ms) " << format_duration(r.setupExperimentMs) << std::endl;
    ofs << "\tPerturb time (ms) " << format_duration(r.perturbExperimentMs) << std::endl;
    ofs << "\tWeighting time (ms) " << format_duration(r.weightingExperimentMs) << std::endl;
    ofs << "\tTotal experiment weight log10: " << std::setprecision(15) << r.experimentWeightLog10 << std::endl;
    ofs << "\tRelative standard error: " << r.relStdError << std::endl;
    ofs << "\tPer-path log10 error bound vs FP64: " << r.weightErrorBoundLog10 << std::endl;
    ofs << "\tRelative error vs FP64 (checked chains): " << r.fp64RelError << std::endl;
    ofs << std::endl;
    return 0;
}
