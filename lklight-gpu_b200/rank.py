"""Reading GSO output and writing ranking lists in the reference's formats.

``parse_gso`` reads a ``gso_<step>.out`` file as ``parse_gso_file`` does
(src/bin/lightdock.rs:123-148): comment and blank lines are skipped, the
values between '(' and the first ')' are the pose (translation, then the
quaternion w, x, y, z, then any ANM extents), and the whitespace-separated
fields after it give the luciferin (third) and the scoring (sixth); the
glowworm id counts every non-comment line, parsable or not.

``write_rank`` writes ``ranking.list``-style files as ``write_rank_file``
does (src/bin/lightdock.rs:888-903): a stable sort by descending scoring
(or luciferin), then one line per solution.  ``rank`` collects the swarms'
files and writes the three lists of ``lklight rank`` (lightdock.rs:905-947;
cluster filtering and the RMSD list are not restated).
"""
import os


def parse_gso(path):
    """Entries of one gso file: dicts with translation, rotation (w, x, y, z),
    luciferin, scoring, glowworm id and extents."""
    out = []
    if not os.path.exists(path):
        return out
    gid = 0
    with open(path) as f:
        for line in f.read().split("\n"):
            s = line.strip()
            if s.startswith("#") or not s:
                continue
            pend = s.find(")")
            if pend >= 0:
                vals = []
                for t in s[1:pend].split(","):
                    try:
                        vals.append(float(t.strip()))
                    except ValueError:
                        pass
                if len(vals) >= 7:
                    rest = s[pend + 1:].split()

                    def num(i):
                        try:
                            return float(rest[i])
                        except (IndexError, ValueError):
                            return 0.0
                    out.append(dict(translation=vals[0:3], rotation=vals[3:7], luciferin=num(2), scoring=num(5),
                                    glowworm=gid, extents=vals[7:]))
            gid += 1
    return out


def collect(num_swarms, steps, directory="."):
    """Solutions of every swarm (collect_solutions, lightdock.rs:863-886)."""
    sols = []
    for sid in range(num_swarms):
        for e in parse_gso(os.path.join(directory, "swarm_%d" % sid, "gso_%d.out" % steps)):
            t = e["translation"]
            sols.append(dict(swarm=sid, glowworm=e["glowworm"], luciferin=e["luciferin"], scoring=e["scoring"],
                             coords="(%.3f,%.3f,%.3f)" % (t[0], t[1], t[2])))
    return sols


def write_rank(solutions, filename, by_scoring=True):
    """One ranking list: stable sort by descending scoring or luciferin."""
    key = "scoring" if by_scoring else "luciferin"
    ranked = sorted(solutions, key=lambda s: -s[key])
    with open(filename, "w") as f:
        f.write("# Rank Swarm Glowworm Luciferin Scoring PDB Coords\n")
        for r, s in enumerate(ranked):
            f.write("%5d %4d %5d %12.6f %12.6f swarm_%d/lightdock_%d.pdb %s\n" % (
                r + 1, s["swarm"], s["glowworm"], s["luciferin"], s["scoring"], s["swarm"], s["glowworm"],
                s["coords"]))
    return ranked


def rank(num_swarms, steps, directory=".", clashes_cutoff=None):
    """ranking.list, rank_by_scoring.list and rank_by_luciferin.list in
    `directory` from its swarm_<i>/gso_<steps>.out files."""
    sols = collect(num_swarms, steps, directory)
    if clashes_cutoff is not None:
        sols = [s for s in sols if s["scoring"] >= clashes_cutoff]
    write_rank(sols, os.path.join(directory, "ranking.list"), True)
    write_rank(sols, os.path.join(directory, "rank_by_scoring.list"), True)
    return write_rank(sols, os.path.join(directory, "rank_by_luciferin.list"), False)
