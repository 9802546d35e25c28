"""Generate the committed golden fixtures for the oracle and parity tests.

Run once in a checkout that has the LKlight-GPU reference sources beside it:
``LKG_REFERENCE`` names their directory, by default ``reference`` next to
this repository's directory.  Nothing at test or bench time reads the
reference: only the files written here do.

Outputs
-------
tests/golden/1azp_models.npz
    Per-atom parameter arrays of the 1AZP receptor and ligand (and each
    atom's residue, for restraint tests), typed the way
    the reference's DNA model (``src/dna.rs:277-403``) and PYDOCK model
    (``src/pydock.rs:41-162``) type them: AMBER type lookup by
    ``RES-ATOM`` with the ``H1/H2/H3 -> RES-H`` and ``*-<element>`` fallbacks,
    electrostatic charge from ``ELE_CHARGES`` then ``NT_ELE_CHARGES`` (else 0),
    vdW well depth / radius by AMBER type (defaults 0.086 / 1.908), heavy flag
    = atom name does not start with ``H``.  The tables are parsed from the
    reference sources here; they are not re-typed.
lklight-gpu_b200/data/amber_types.json
    The DNA family's 54-entry vdW type table (``src/dna.rs:88-105``) and the
    DA/DC/DG/DT atom-name -> AMBER-type maps (``src/dna.rs:117-132``) that the
    synthetic complex generator draws from.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("LKG_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))


def parse_tables(path):
    """Parse every ``static ref NAME: HashMap<..> = hashmap![k => v, ...];``.

    Later duplicate keys overwrite earlier ones, as ``HashMap::insert`` does.
    """
    src = open(path).read()
    out = {}
    for name, body in re.findall(
            r'static ref (\w+): HashMap<[^>]*> = hashmap!\[(.*?)\];', src, re.S):
        table = {}
        for k, v in re.findall(r'"([^"]*)"\s*=>\s*("[^"]*"|[^,\]\s]+)', body):
            table[k] = v.strip('"') if v.startswith('"') else float(v)
        out[name] = table
    return out


def parse_pdb(path):
    """Fixed-column PDB ATOM/HETATM reader (file order, as pdbtbx keeps it)."""
    atoms = []
    for line in open(path):
        if not line.startswith(("ATOM", "HETATM")):
            continue
        atoms.append(dict(
            name=line[12:16].strip(), res=line[17:20].strip(),
            chain=line[21], resseq=int(line[22:26]), icode=line[26].strip(),
            x=float(line[30:38]), y=float(line[38:46]), z=float(line[46:54]),
            element=line[76:78].strip()))
    return atoms


def type_atoms(atoms, t, with_heavy):
    """Restates the typing loop of ``DNADockingModel::new`` (src/dna.rs:335-399)
    and ``PYDOCKDockingModel::new`` (src/pydock.rs:107-155)."""
    amber, ele, nt = t["AMBER_TYPES"], t["ELE_CHARGES"], t["NT_ELE_CHARGES"]
    vc, vr = t["VDW_CHARGES"], t["VDW_RADII"]
    coords, q, eps, rad, heavy = [], [], [], [], []
    for a in atoms:
        res, name = a["res"], a["name"]
        atom_id = f"{res}-{name}"
        if atom_id in amber:
            at = amber[atom_id]
        else:
            h_id = f"{res}-H"
            if name in ("H1", "H2", "H3") and h_id in amber:
                atom_id = h_id
                at = amber[atom_id]
            else:
                elem = (name[:1] or "C").upper()
                atom_id = f"*-{elem}"
                at = amber.get(atom_id, "C")
        charge = ele.get(atom_id, nt.get(atom_id, 0.0))
        coords.append((a["x"], a["y"], a["z"]))
        q.append(charge)
        eps.append(vc.get(at, 0.086))
        rad.append(vr.get(at, 1.908))
        heavy.append(0 if name.startswith("H") else 1)
    d = dict(coords=np.array(coords, np.float64), ele=np.array(q, np.float64),
             vdw=np.array(eps, np.float64), radius=np.array(rad, np.float64))
    if with_heavy:
        d["heavy"] = np.array(heavy, np.uint8)
    return d


def main():
    dna_t = parse_tables(os.path.join(REF, "src/dna.rs"))
    amb_t = parse_tables(os.path.join(REF, "src/amber.rs"))
    rec = parse_pdb(os.path.join(REF, "tests/1azp/1azp_receptor.pdb"))
    lig = parse_pdb(os.path.join(REF, "tests/1azp/1azp_ligand.pdb"))
    arrays = {}
    for fam, tables, hv in (("dna", dna_t, True), ("pydock", amb_t, False)):
        for side, atoms in (("rec", rec), ("lig", lig)):
            for k, v in type_atoms(atoms, tables, hv).items():
                arrays[f"{fam}_{side}_{k}"] = v
    # element-column hydrogen flag (cpydock typing, src/cpydock.rs:263-266)
    for side, atoms in (("rec", rec), ("lig", lig)):
        arrays[f"{side}_is_h"] = np.array(
            [1 if (a["element"] == "H" if a["element"] else a["name"].startswith("H"))
             else 0 for a in atoms], np.uint8)
    # residue of every atom: dense index (first appearance) and the id the
    # reference keys its restraint maps by, "chain.resname.serial[icode]"
    # (src/pydock.rs:66-69)
    for side, atoms in (("rec", rec), ("lig", lig)):
        ids, index = [], {}
        per_atom = []
        for a in atoms:
            rid = f"{a['chain']}.{a['res']}.{a['resseq']}{a['icode']}"
            if rid not in index:
                index[rid] = len(ids)
                ids.append(rid)
            per_atom.append(index[rid])
        arrays[f"{side}_resid"] = np.array(per_atom, np.int32)
        arrays[f"{side}_residues"] = np.array(ids)
    np.savez_compressed(os.path.join(HERE, "1azp_models.npz"), **arrays)

    # DNA-family vdW type table + nucleotide maps for the synthetic generator.
    types = sorted(dna_t["VDW_CHARGES"].keys())
    table = {
        "source": "src/dna.rs:88-105 (VDW_CHARGES, VDW_RADII), src/dna.rs:117-132 (AMBER_TYPES D*)",
        "types": [[k, dna_t["VDW_CHARGES"][k], dna_t["VDW_RADII"][k]] for k in types],
        "nucleotides": {},
    }
    for nuc in ("DA", "DC", "DG", "DT"):
        table["nucleotides"][nuc] = [
            [k.split("-", 1)[1], v] for k, v in dna_t["AMBER_TYPES"].items()
            if k.startswith(nuc + "-")]
    with open(os.path.join(REPO, "lklight-gpu_b200", "data", "amber_types.json"), "w") as f:
        json.dump(table, f, indent=1)
    print("wrote", len(arrays), "arrays;", len(types), "types")


if __name__ == "__main__":
    sys.exit(main())
