"""calcPhiASE -- command-line entry point with the reference executable's shape.

Same three flags and error behaviour as the reference's ``calcPhiASE``
(src/openpmd_main.cpp:30-122): ``--input-path=<file>``, ``--output-path=<file>``
and ``--cpp-control``; any other argument is rejected as unsupported; on
failure ``calcPhiASE failed: <what>`` goes to stderr and the exit code is 1.

The input is an ``.npz`` request whose record and attribute names follow the
reference's openPMD schema (pyInclude/openpmd/schema/builtins.py:21-198):
``points``/``connectivity``/``numberOfLevels``/``thickness``/``betaVolume``/
``betaCells``/``claddingCellType``/``claddingNumber``/``claddingAbsorption``/
``nTot``/``crystalTFluo``/``reflectivity``/``refractiveIndex``,
``lambdaAbsorption``/``sigmaAbsorption``/``lambdaEmission``/``sigmaEmission``/
``spectralResolution``/``monochromatic`` and the controls ``minRays``/
``maxRays``/``relativeStandardErrorThreshold``/``repetitions``/
``adaptiveSteps``/``useReflections``/``minSampleRange``/``maxSampleRange``/
``rngSeed``/``propagationMode``.  The output ``.npz`` holds the result
records ``phiAse``/``standardError``/``relativeStandardError``/``totalRays``/
``dndtAse``/``droppedRays`` and the reflection metadata attributes.
(openPMD-api is not available to this build, hence the npz container.)
"""

from __future__ import annotations

import sys

import numpy as np


class CliError(RuntimeError):
    pass


def parse_paths(argv):
    paths = {"input": None, "output": None, "cppControl": False}
    for arg in argv:
        if arg.startswith("--input-path="):
            paths["input"] = arg[len("--input-path="):]
        elif arg.startswith("--output-path="):
            paths["output"] = arg[len("--output-path="):]
        elif arg == "--cpp-control":
            paths["cppControl"] = True
        else:
            raise CliError(f"Unsupported argument '{arg}'. calcPhiASE only accepts --input-path, --output-path, "
                           "and --cpp-control.")
    if not paths["input"]:
        raise CliError("Missing required --input-path=<request.npz>.")
    if not paths["output"]:
        raise CliError("Missing required --output-path=<result.npz>.")
    return paths


def _scalar(d, name, default=None, cast=float):
    if name in d.files:
        return cast(np.asarray(d[name]).ravel()[0])
    if default is None:
        raise CliError(f"request is missing required attribute '{name}'")
    return default


def _array(d, name, required=True):
    if name in d.files:
        return np.asarray(d[name])
    if required:
        raise CliError(f"request is missing required record '{name}'")
    return None


def request_from_npz(path):
    from .mesh import PrismMesh
    from .simulation import PhiASE
    from .spectra import CrossSectionData

    d = np.load(path, allow_pickle=False)
    if "mseThreshold" in d.files:
        raise CliError("mseThreshold is not a request attribute; use relativeStandardErrorThreshold")
    mesh = PrismMesh(
        points=_array(d, "points"), triangles=_array(d, "connectivity"),
        numberOfLevels=_scalar(d, "numberOfLevels", cast=int), thickness=_scalar(d, "thickness"),
        betaVolume=_array(d, "betaVolume"), nTot=_scalar(d, "nTot"), crystalTFluo=_scalar(d, "crystalTFluo"),
        betaCells=_array(d, "betaCells", False), claddingCellTypes=_array(d, "claddingCellType", False),
        claddingNumber=_scalar(d, "claddingNumber", 1, int), claddingAbsorption=_scalar(d, "claddingAbsorption", 0.0),
        reflectivities=_array(d, "reflectivity", False), refractiveIndices=_array(d, "refractiveIndex", False))
    sa = _array(d, "sigmaAbsorption")
    se = _array(d, "sigmaEmission")
    la = _array(d, "lambdaAbsorption", False)
    le = _array(d, "lambdaEmission", False)
    spectra = CrossSectionData(la if la is not None else np.arange(sa.size, dtype=float), sa,
                               le if le is not None else np.arange(se.size, dtype=float), se,
                               _scalar(d, "spectralResolution", max(sa.size, se.size), int))
    mode = str(d["propagationMode"]) if "propagationMode" in d.files else "backward"
    phi = PhiASE(
        propagationMode=mode, minRays=_scalar(d, "minRays", cast=int),
        maxRays=_scalar(d, "maxRays", _scalar(d, "minRays", cast=int), int),
        relativeStandardErrorThreshold=_scalar(d, "relativeStandardErrorThreshold", 0.0),
        repetitions=_scalar(d, "repetitions", 1, int), adaptiveSteps=_scalar(d, "adaptiveSteps", 0, int),
        useReflections=bool(_scalar(d, "useReflections", 0, int)),
        monochromatic=bool(_scalar(d, "monochromatic", 0, int)),
        minSampleRange=_scalar(d, "minSampleRange", 0, int),
        maxSampleRange=_scalar(d, "maxSampleRange", mesh.numberOfSamples - 1, int),
        rngSeed=_scalar(d, "rngSeed", 5489, int))
    return phi, mesh, spectra


def write_result(path, result):
    np.savez(path, phiAse=result.phiAse, standardError=result.standardError,
             relativeStandardError=result.relativeStandardError, totalRays=result.totalRays, dndtAse=result.dndtAse,
             droppedRays=result.droppedRays, srmStatus=np.asarray(result.srmStatus),
             srmPasses=np.uint32(result.srmPasses), srmRemainingFraction=np.float64(result.srmRemainingFraction),
             srmMaxIterations=np.uint32(result.srmMaxIterations),
             srmDivergenceStreak=np.uint32(result.srmDivergenceStreak))


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    try:
        paths = parse_paths(argv)
        if paths["cppControl"]:
            raise CliError("--cpp-control (compiled time-stepped simulation) is not provided by this build")
        phi, mesh, spectra = request_from_npz(paths["input"])
        result = phi.run(gainMedium=mesh, crossSections=spectra).getResults()
        write_result(paths["output"], result)
        return 0
    except Exception as exc:  # mirror the reference: one line, exit code 1
        print(f"calcPhiASE failed: {exc}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
