"""Generates the golden fixtures: small .conf/.pro cases and the output files
the flysim reference writes for them.

The reference is built from its own sources by oracle/Makefile.ref into
oracle/_ref/flysim_ref (this needs the reference tree, so it runs only where
the sources are; the fixtures are committed).  Each case directory holds
net.conf, net.pro, cmd (the reference's extra command-line flags) and the
reference's output files; the two log files it writes on every run
(ConfsInfo.log, network.log) are recorded as size and SHA-256 in logs.json.

    python tests/golden/make_golden.py              # all cases from scratch
    python tests/golden/make_golden.py --logs-only  # logs.json of the committed cases
    python tests/golden/make_golden.py --case NAME  # one case (or several names)

Cases at the benchmark configurations keep digests instead of files:
config1_1s (the two-population E=800 / I=200 network of the plain method
for its full 1 s) records the size and SHA-256 of every output file in
digests.json; connectome20k_d0 (the 20,000-neuron connectome-shaped network
with delays 0, 100 ms, reference run with -t 1) does the same and does not
keep its 354 MB net.conf either: gen.json names the seeded generator call
that rewrites it and the SHA-256 the rewritten file must have.
"""
from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from flysim_b200 import netgen  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "flysim_ref")

OUTS = [{"name": "Spikes.dat", "type": "Spike", "pop": "AllPopulation"},
        {"name": "FR.dat", "type": "FiringRate", "pop": "AllPopulation", "win": 50, "step": 10},
        {"name": "FRs.dat", "type": "FiringRate", "pop": "AllPopulation", "win": 20, "step": 5, "sum": True}]


def _misc_conf(path):
    s = ""
    for name, n in (("A", 30), ("B", 20), ("C", 1), ("D", 1)):
        s += ("NeuralPopulation: %s\nN=%d\nC=0.5\nTaum=15\nRestPot=-65\nThreshold=-50\nResetPot=-60\n"
              "RefractoryPeriod=2.5\nSpikeDly=0.3\n\n"
              "Receptor:AMPA\nTau=3\nRevPot=0\nFreqExt=3000\nMeanExtEff=2.5\nEndReceptor\n\n"
              "Receptor:Ach\nTau=4\nRevPot=0\nFreqExt=200\nMeanExtEff=1\nEndReceptor\n\n"
              "Receptor:GluCl\nTau=6\nRevPot=-80\nFreqExt=100\nMeanExtEff=1\nEndReceptor\n\n"
              "Receptor:GABA\nTau=5\nRevPot=-70\nEndReceptor\n\n"
              "Receptor:NMDA\nTau=80\nTauXT=2\nRevPot=0\nFreqExt=50\nMeanExtEff=0.5\nEndReceptor\n\n") % (name, n)
        links = {
            "A": [("B", "Ach", 0.4, 0.3, None), ("A", "GAP", 0.01, 0.2, None), ("C", "GAP", 0.02, None, None),
                  ("B", "NMDA", 0.1, 0.5, None)],
            "B": [("A", "GluCl", 0.5, 0.03, None), ("A", "GABA", 1.5, 0.05, None), ("D", "Ach", 3, None, None),
                  ("A", "Ach", 3, 0.5, 0.5)],
            "C": [("D", "GAP", 0.05, None, None), ("A", "AMPA", 5, 0.5, None)],
            "D": [],
        }[name]
        for tgt, rec, eff, conn, wgt in links:
            s += "TargetPopulation: %s\nTargetReceptor=%s\nMeanEff=%s\n" % (tgt, rec, eff)
            if conn is not None:
                s += "Connectivity=%s\n" % conn
            if wgt is not None:
                s += "weight=%s\n" % wgt
            s += "EndTargetPopulation\n\n"
        s += "EndNeuralPopulation\n\n"
    with open(path, "w") as f:
        f.write(s)


def _small_conf(path):
    """Two 20-neuron populations with short-term plasticity parameters,
    spike delay and a self-connected group."""
    s = ""
    for name, selfc in (("Exc1", False), ("Exc2", True)):
        s += ("NeuralPopulation: %s\nN=20\nC=0.5\nTaum=20\nThreshold=-50\nRestPot=-70\nResetPot=-55\n"
              "RefractoryPeriod=1.9\nSpikeDly=0.3\n" % name)
        if name == "Exc1":
            s += "STP_pv=0.6\nSTP_tD=300\nSTP_aF=1.0\nSTP_tF=7000\nSTP_aCap=2.0\nSTP_tCap=100\nSTP_aCar=3.0\nSTP_tCar=70\n"
        if selfc:
            s += "SelfConnection=true\n"
        s += "\nReceptor:AMPA\nTau=5\nRevPot=-70\nFreqExt=8.4375\nMeanExtEff=2.1\nEndReceptor\n\n"
        s += "TargetPopulation: Exc2\nTargetReceptor=AMPA\nMeanEff=4.2\n"
        if name == "Exc1":
            s += "Connectivity=0.5\n"
        s += "EndTargetPopulation\n\nEndNeuralPopulation\n\n"
    with open(path, "w") as f:
        f.write(s)


def _keywords_case(d):
    """Less common keywords: LeakyConductance (shown in ConfsInfo.log only),
    MeanExtCon, the LTP_* parameters (with -LTP, on single-target records),
    a CurrentInjec event on a group, the SubType keyword, a group output."""
    recs = ("Receptor:AMPA\nTau=3\nRevPot=0\nFreqExt=2500\nMeanExtEff=2.0\nMeanExtCon=1.5\nEndReceptor\n\n"
            "Receptor:GABA\nTau=5\nRevPot=-70\nEndReceptor\n\n"
            "Receptor:NMDA\nTau=80\nTauXT=2\nRevPot=0\nEndReceptor\n\n")
    conf = ""
    for name, n, extra, links in (
            ("P", 30, "LeakyConductance=20\nLTP_tLP=30\nLTP_SpiLPDy=2\nLTP_PosISI=0.02\nLTP_NegISI=-0.01\n",
             (("Q", "AMPA", 1.5, 0.02), ("Q", "NMDA", 0.3, 0.02), ("P", "AMPA", 0.2, 0.3))),
            ("Q", 20, "", (("P", "GABA", 2, 0.5), ("P", "AMPA", 1.0, 0.01)))):
        conf += ("NeuralPopulation: %s\nN=%d\nC=0.5\nTaum=15\nRestPot=-65\nThreshold=-50\nResetPot=-60\n"
                 "RefractoryPeriod=2\nSpikeDly=0.5\n%s\n%s") % (name, n, extra, recs)
        for tgt, rec, eff, conn in links:
            conf += ("TargetPopulation: %s\nTargetReceptor=%s\nMeanEff=%s\nConnectivity=%s\n"
                     "EndTargetPopulation\n\n") % (tgt, rec, eff, conn)
        conf += "EndNeuralPopulation\n\n"
    with open(os.path.join(d, "net.conf"), "w") as f:
        f.write(conf)
    pro = ("DefineMacro\nGroupName:PQ\nGroupMembers:P,Q\nEndGroupMembers\nRandomSeeds: 77\nEndRandomSeeds\n"
           "EndDefineMacro\n\n"
           "EventTime 40\nType=CurrentInjec\nLabel=inj\nPopulation: PQ\nGaussMean=0.2\nGaussSTD=0.5\nEndEvent\n\n"
           "EventTime 80\nType=ChangeExtFreq\nLabel=#2#\nPopulation: Q\nSubType: AMPA\nFreqExt=0\nEndEvent\n\n"
           "EventTime 150\nType=EndTrial\nLabel=End_of_the_trial\nEndEvent\n\n"
           "OutControl\nFileName:Spikes.dat\nType=Spike\npopulation:AllPopulation\nEndOutputFile\n\n"
           "FileName:FR.dat\nType=FiringRate\nFiringRateWindow=20\nPrintStep=10\npopulation:PQ\nEndOutputFile\n\n"
           "EndOutControl\n")
    with open(os.path.join(d, "net.pro"), "w") as f:
        f.write(pro)


def cases():
    c = {}
    c["two_pop"] = dict(conf=lambda p: netgen.write_two_pop(p),
                        pro=dict(t_end_ms=200, seeds=(7,), outputs=OUTS), flags=[])
    c["two_pop_std"] = dict(conf=lambda p: netgen.write_two_pop(p, n_e=200, n_i=50),
                            pro=dict(t_end_ms=150, seeds=(3,), outputs=OUTS), flags=["-STD"])
    c["two_pop_stp"] = dict(conf=lambda p: netgen.write_two_pop(p, n_e=200, n_i=50),
                            pro=dict(t_end_ms=150, seeds=(3,), outputs=OUTS), flags=["-STP"])

    def conn_ltp(p):
        netgen.write_connectome(netgen.connectome(n=150, regions=5, mean_degree=20, delays=False, seed=5), p,
                                with_delays=False)
    c["conn_ltp"] = dict(conf=conn_ltp, pro=dict(t_end_ms=200, seeds=(4,), outputs=OUTS), flags=["-LTP"])

    # LTP keywords strong enough to move the weights within a trial, and two
    # repeats: the reference's VarInit leaves the records' weights as LTP
    # left them (code/EqsGnl2.cpp:339-401), so the second trial starts from
    # the first trial's weights
    def ltp_repeats(p):
        netgen.write_connectome(netgen.connectome(n=150, regions=5, mean_degree=20, delays=False, seed=8), p,
                                with_delays=False, ltp=dict(tLP=30, SpiLPDy=0.2, PosISI=0.05, NegISI=-0.02))
    c["ltp_repeats"] = dict(conf=ltp_repeats, pro=dict(t_end_ms=150, seeds=(4, 6), outputs=OUTS),
                            flags=["-LTP", "-rp", "2"])

    def conn(p):
        netgen.write_connectome(netgen.connectome(n=400, regions=8, mean_degree=40, delays=False, seed=2), p,
                                with_delays=False)
    c["conn"] = dict(conf=conn, pro=dict(t_end_ms=200, seeds=(11,), outputs=OUTS + [
        {"name": "Isyn.dat", "type": "IsynSeparatedSum", "pop": ["n3", "n7"]},
        {"name": "ov.dat", "type": "DeltaMemPotLimit", "pop": "AllPopulation", "align": True},
        {"name": "gv.dat", "type": "GatingVariable", "pop": "n1"}]), flags=[])
    c["repeats"] = dict(conf=lambda p: netgen.write_two_pop(p, n_e=160, n_i=40), pro=dict(
        t_end_ms=100, seeds=(5, 9), outputs=OUTS,
        events=[{"t": 30, "type": "ChangeExtFreq", "pop": "E", "f": 0},
                {"t": 50, "type": "ChangeMembraneNoise", "pop": "AllPopulation", "mean": 0.2, "std": 0.5},
                {"t": 70, "type": "ChangeExtFreq", "pop": "I", "rec": "NMDA", "f": 300}]), flags=["-rp", "3"])
    c["misc"] = dict(conf=_misc_conf, pro=dict(t_end_ms=200, seeds=(21,), outputs=OUTS + [
        {"name": "Isyn.dat", "type": "IsynSeparatedSum", "pop": ["C", "D"]},
        {"name": "ov.dat", "type": "DeltaMemPotLimit", "pop": "AllPopulation"},
        {"name": "sa.dat", "type": "Spike", "pop": ["B", "A"], "align": True},
        {"name": "Mem.dat", "type": "MemPot", "pop": ["D", "C"]}],
        events=[{"t": 100, "type": "ChangeExtFreq", "pop": "A", "rec": "Ach", "f": 0},
                {"t": 150, "type": "ChangeMembraneNoise", "pop": "B", "mean": 0.3, "std": 2.0}]), flags=[])
    c["small"] = dict(conf=_small_conf, pro=dict(
        t_end_ms=1000, seeds=(12345,), groups={"Sti2": ["Exc2", "Exc1"]},
        outputs=[{"name": "Spikes.dat", "type": "Spike", "pop": "Sti2"},
                 {"name": "FRates.dat", "type": "FiringRate", "pop": "Exc2", "win": 50, "step": 10}],
        events=[{"t": 300, "type": "ChangeExtFreq", "pop": "Exc1", "f": 24000},
                {"t": 650, "type": "ChangeMembraneNoise", "pop": "Exc1", "mean": 0.43, "std": 0.03}]), flags=[])
    c["keywords"] = dict(raw=_keywords_case, flags=["-LTP"])
    # the benchmark configurations themselves (digests only)
    c["config1_1s"] = dict(conf=lambda p: netgen.write_two_pop(p), pro=dict(t_end_ms=1000, seeds=(7,), outputs=OUTS),
                           flags=[], digests=True)
    c["connectome20k_d0"] = dict(gen=dict(n=20000, regions=58, seed=1), pro=dict(
        t_end_ms=100, seeds=(1,), outputs=OUTS[:2]), flags=["-t", "1"], digests=True)
    # command-line options: user seed (which also switches STD on, as the
    # reference's flag parser does), a non-default time step, and the
    # -om / -os / -or outputs added on top of the .pro's
    c["cli_flags"] = dict(conf=lambda p: netgen.write_two_pop(p, n_e=16, n_i=8), pro=dict(
        t_end_ms=40, seeds=(5,), outputs=OUTS[:1]),
        flags=["-udfsed", "7", "-dt", "0.05", "-om", "m.dat", "-os", "s.dat", "-or", "r.dat"])
    return c


LOGS = ("ConfsInfo.log", "network.log")


def write_generated_conf(gen: dict, path: str) -> None:
    """The .conf of a generated case: connectome-shaped network, delays 0."""
    c = netgen.connectome(n=gen["n"], regions=gen["regions"], seed=gen["seed"])
    netgen.write_connectome(c, path, with_delays=False)


def file_record(path: str) -> dict:
    h = hashlib.sha256()
    size = lines = 0
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 22), b""):
            h.update(block)
            size += len(block)
            lines += block.count(b"\n")
    return {"bytes": size, "lines": lines, "sha256": h.hexdigest()}


def record_digests(d, keep=("net.conf", "net.pro", "cmd.json", "logs.json", "gen.json")):
    """Replaces the output files in d by their sizes and SHA-256 (digests.json)."""
    rec = {}
    for f in sorted(os.listdir(d)):
        if f in keep or f == "digests.json":
            continue
        rec[f] = file_record(os.path.join(d, f))
        os.remove(os.path.join(d, f))
    with open(os.path.join(d, "digests.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


def record_logs(d):
    """Replaces the reference's log files in d by their digests (logs.json)."""
    rec = {}
    for f in LOGS:
        p = os.path.join(d, f)
        data = open(p, "rb").read()
        rec[f] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
        os.remove(p)
    with open(os.path.join(d, "logs.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


def record_threaded_log(d, flags):
    """Adds to logs.json the digest of the network.log the reference writes
    with -t 4: set-up draws depend on the thread count (the run itself is
    not reproducible with several threads, its set-up is)."""
    with tempfile.TemporaryDirectory() as t:
        for f in ("net.conf", "net.pro"):
            shutil.copy(os.path.join(d, f), t)
        r = subprocess.run([REF, "-conf", "net.conf", "-pro", "net.pro"] + flags + ["-t", "4"], cwd=t,
                           capture_output=True, text=True)
        if r.returncode != 0:
            sys.exit("reference failed on %s -t 4: %s" % (d, r.stderr[-400:]))
        data = open(os.path.join(t, "network.log"), "rb").read()
    p = os.path.join(d, "logs.json")
    rec = json.load(open(p))
    rec["network.log -t 4"] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(p, "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)


def logs_only():
    for name in sorted(os.listdir(HERE)):
        d = os.path.join(HERE, name)
        if not os.path.isfile(os.path.join(d, "cmd.json")):
            continue
        flags = json.load(open(os.path.join(d, "cmd.json")))
        with tempfile.TemporaryDirectory() as t:
            for f in ("net.conf", "net.pro"):
                shutil.copy(os.path.join(d, f), t)
            r = subprocess.run([REF, "-conf", "net.conf", "-pro", "net.pro"] + flags, cwd=t,
                               capture_output=True, text=True)
            if r.returncode != 0:
                sys.exit("reference failed on %s: %s" % (name, r.stderr[-400:]))
            record_logs(t)
            shutil.copy(os.path.join(t, "logs.json"), d)
        record_threaded_log(d, flags)
        print(name, open(os.path.join(d, "logs.json")).read().replace("\n", " "))


def main():
    if not os.path.exists(REF):
        sys.exit("reference binary missing: build it with  make -f oracle/Makefile.ref")
    if "--logs-only" in sys.argv:
        return logs_only()
    only = sys.argv[sys.argv.index("--case") + 1:] if "--case" in sys.argv else None
    for name, cs in cases().items():
        if only and name not in only:
            continue
        d = os.path.join(HERE, name)
        shutil.rmtree(d, ignore_errors=True)
        os.makedirs(d)
        if "raw" in cs:
            cs["raw"](d)
        elif "gen" in cs:
            write_generated_conf(cs["gen"], os.path.join(d, "net.conf"))
            netgen.write_pro(os.path.join(d, "net.pro"), **cs["pro"])
            with open(os.path.join(d, "gen.json"), "w") as f:
                json.dump(dict(cs["gen"], conf=file_record(os.path.join(d, "net.conf"))), f, indent=1, sort_keys=True)
        else:
            cs["conf"](os.path.join(d, "net.conf"))
            netgen.write_pro(os.path.join(d, "net.pro"), **cs["pro"])
        with open(os.path.join(d, "cmd.json"), "w") as f:
            json.dump(cs["flags"], f)
        r = subprocess.run([REF, "-conf", "net.conf", "-pro", "net.pro"] + cs["flags"], cwd=d,
                           capture_output=True, text=True)
        if r.returncode != 0:
            sys.exit("reference failed on %s: %s" % (name, r.stderr[-400:]))
        record_logs(d)
        if "gen" not in cs:  # a second parse of a generated network is minutes of reference time
            record_threaded_log(d, cs["flags"])
        if cs.get("digests"):
            record_digests(d)
        if "gen" in cs:
            os.remove(os.path.join(d, "net.conf"))
        outs = sorted(f for f in os.listdir(d) if f not in ("net.conf", "net.pro", "cmd.json", "logs.json"))
        print(name, outs)


if __name__ == "__main__":
    main()
