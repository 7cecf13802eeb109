"""In-process hampyx: the reference's Python wrapper interface
(hampyx/hampyx.py) running the B200 integrator in the calling process
instead of a ``hamx`` subprocess.

    import hammurabix_b200.hampyx as hpx
    obj = hpx.Hampyx(xml_path="params.xml")          # exe_path not needed
    obj.mod_par(keychain=["observable", "sync"], attrib={"freq": "30"})
    obj()                                             # run
    obj.sim_map[("sync", "30", "32", "Q")]            # numpy map

``sim_map`` keys are the reference's: (kind, freq string as in the XML,
nside string, 'I'|'Q'|'U'|'nan') (hampyx.py:52-60, 306-338).  The XML
editing methods follow hampyx.py:364-470.  ``precision`` selects the FP64
parity form (default) or the FP32-compensated form.
"""
import os
import tempfile
import xml.etree.ElementTree as et

from .integrator import Integrator
from .pipeline import Pipeline


class Hampyx:
    def __init__(self, xml_path=None, exe_path=None, precision="fp64", device=0):
        self.wk_dir = os.getcwd()
        if xml_path is None:
            cand = [s for s in os.listdir(self.wk_dir) if "xml" in s]
            cand = [os.path.join(self.wk_dir, c) for c in cand
                    if os.path.isfile(os.path.join(self.wk_dir, c))]
            if not cand:
                raise ValueError("no XML parameter file found in the working directory")
            xml_path = cand[0]
        self.xml_path = os.path.abspath(xml_path)
        if not os.path.isfile(self.xml_path):
            raise ValueError(f"missing XML file {self.xml_path}")
        self.exe_path = exe_path  # kept for interface compatibility; unused
        self.tree = et.parse(self.xml_path)
        self.sim_map = {}
        self.precision = precision
        self._integ = Integrator(precision, device=device)

    def __call__(self, verbose=False):
        return self.run(verbose)

    def run(self, verbose=False):
        """Run the LOS integration of the (edited) parameter tree and fill
        sim_map (hampyx.py:232-267)."""
        fd, path = tempfile.mkstemp(prefix="params_", suffix=".xml", dir=self.wk_dir)
        os.close(fd)
        try:
            self.tree.write(path)
            pipe = Pipeline(path, integrator=self._integ)
            maps = pipe.run()
        finally:
            os.remove(path)
        self.sim_map.update(maps)
        if verbose:
            for k, v in maps.items():
                print(k, v.shape, float(abs(v).max()))
        return self.sim_map

    # ---- XML manipulation: hampyx.py:364-470 -------------------------------
    @staticmethod
    def _path(keychain):
        return "./" + "/".join(keychain)

    def mod_par(self, keychain=None, attrib=None):
        if type(attrib) is not dict or type(keychain) is not list:
            raise ValueError("wrong input %s %s" % (keychain, attrib))
        target = self.tree.getroot().find(self._path(keychain))
        if target is None:
            raise ValueError("wrong path %s" % self._path(keychain))
        for k, v in attrib.items():
            target.set(k, v)

    def add_par(self, keychain=None, subkey=None, attrib=None):
        if type(keychain) is not list or type(subkey) is not str:
            raise ValueError("wrong input %s %s %s" % (keychain, subkey, attrib))
        target = self.tree.getroot().find(self._path(keychain))
        if target is None:
            raise ValueError("wrong path %s" % self._path(keychain))
        if attrib is None:
            et.SubElement(target, subkey)
        elif type(attrib) is dict:
            for existed in target.findall(subkey):
                if existed.attrib == attrib:
                    raise ValueError("repeatitive input %s %s %s" % (keychain, subkey, attrib))
            et.SubElement(target, subkey, attrib)
        else:
            raise ValueError("wrong input %s %s %s" % (keychain, subkey, attrib))

    def print_par(self, keychain=None):
        root = self.tree.getroot()
        if keychain is None:
            for child in root:
                print(child.tag, child.attrib)
            return
        if type(keychain) is not list:
            raise ValueError("wrong input %s" % keychain)
        for target in root.findall(self._path(keychain)):
            print(target.tag, target.attrib)
            for child in target:
                print("|--> ", child.tag, child.attrib)

    def del_par(self, keychain=None, opt=None):
        if type(keychain) is not list or not keychain:
            raise ValueError("wrong input %s" % keychain)
        root = self.tree.getroot()
        path = self._path(keychain)
        parent = root.find(self._path(keychain[:-1])) if len(keychain) > 1 else root
        target = root.find(path)
        if target is None or parent is None:
            raise ValueError("wrong path %s" % path)
        if opt is None:
            parent.remove(target)
        elif opt == "all":
            for t in root.findall(path):
                parent.remove(t)
        else:
            raise ValueError("unsupported option at %s" % keychain)
