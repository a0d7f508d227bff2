"""Parameter and data-group checks of the imaging drivers.

Drop-in for src/astroviper/utils/check_params.py: check_params (:4-189) and
check_sel_params (:229-347), with the reference's return values, defaults
written into the caller's dict, printed messages and assertion texts (callers
and users read them).  check_sel_params works on an xarray Dataset or any
object with ``data_vars`` and ``attrs["data_groups"]``.
"""
import copy

import numpy as np

_ERR = "######### ERROR:Parameter "


def _is_one_of(x, types):
    return any(isinstance(x, t) for t in types)


def _check_value(key, value, acceptable_data, acceptable_range):
    """The value / range tests shared by scalars and list elements."""
    if acceptable_data is not None and value not in acceptable_data:
        print("######### ERROR: Invalid", key, ". Can only be one of ", acceptable_data, ".")
        return False
    if acceptable_range is not None and (value < acceptable_range[0]
                                         or value > acceptable_range[1]):
        print("######### ERROR: Invalid", key, ". Must be within the range ",
              acceptable_range, ".")
        return False
    return True


def check_params(parm_dict, string_key, acceptable_data_types, acceptable_data=None,
                 acceptable_range=None, list_acceptable_data_types=None, list_len=None,
                 default=None):
    """Checks parm_dict[string_key] (utils/check_params.py:4-189); returns
    whether it passes.  A missing key takes `default` (written into
    parm_dict) or fails when there is none.  A key whose acceptable types
    include list or np.array is checked as a sequence: its length against
    list_len (-1: any) and every element against list_acceptable_data_types,
    acceptable_data and acceptable_range.  A dict-typed key fills its missing
    entries from `default` and checks the others against their defaults'
    types; as in the reference, it then passes whatever those checks found.
    Any other key is checked as a scalar."""
    if string_key not in parm_dict:
        if default is None:
            print(_ERR, string_key, "must be specified")
            return False
        parm_dict[string_key] = default
        return True
    value = parm_dict[string_key]
    if list in acceptable_data_types or np.array in acceptable_data_types:
        if list_len != -1 and len(value) != list_len:
            print(_ERR, string_key, "must be a list of ", list_acceptable_data_types,
                  " and length", list_len, ". Wrong length.")
            return False
        for x in value:
            if not _is_one_of(x, list_acceptable_data_types):
                print(_ERR, string_key, "must be a list of ", list_acceptable_data_types,
                      " and length", len(value), ". Wrong type of", type(x))
                return False
            if not _check_value(string_key, x, acceptable_data, acceptable_range):
                return False
        return True
    if dict in acceptable_data_types:
        if default is None:
            print("######### ERROR:Dictionary parameters must have a default. "
                  "Please report bug.")
            return False
        for k, d in default.items():
            if k in value:
                check_params(value, k, [type(d)], default=d)
            else:
                value[k] = d
        return True
    if not _is_one_of(value, acceptable_data_types):
        print(_ERR, string_key, "must be of type ", acceptable_data_types)
        return False
    return _check_value(string_key, value, acceptable_data, acceptable_range)


def check_sel_params(xds, sel_params, default_data_group_in_name=None,
                     default_data_group_out_name=None, default_data_group_out_modified=None):
    """Input and output data groups of a selection (utils/check_params.py:
    229-347): (data_group_in, data_group_out), the latter merged over the
    former.  With sel_params["overwrite"] (default False) the data groups of
    xds that share a variable with the output group are removed from
    xds.attrs["data_groups"]; without it an output variable that xds already
    holds fails an assertion."""
    modified = {} if default_data_group_out_modified is None else default_data_group_out_modified
    dv_names = list(xds.data_vars)
    groups = copy.deepcopy(xds.attrs.get("data_groups", {}))
    name_in = sel_params.get("data_group_in_name")
    if name_in is not None:
        assert name_in in groups, ("Data group " + name_in +
                                   " not found in xds data_groups: " + str(groups.keys()))
    else:
        name_in = default_data_group_in_name
        assert name_in in groups, ("Default data group " + name_in +
                                   " not found in xds data_groups: " + str(groups.keys()))
    group_in = groups[name_in]
    group_in["data_group_in_name"] = name_in
    # the output group: as given, else the modified defaults; its name as
    # given, else the default name
    group_out = sel_params["data_group_out"] if "data_group_out" in sel_params else modified
    group_out["data_group_out_name"] = sel_params.get("data_group_out_name",
                                                      default_data_group_out_name)
    group_out = {**modified, **group_out}
    sel_params.setdefault("overwrite", False)
    if sel_params["overwrite"]:
        out_values = set(group_out.values())
        for gname, g in groups.items():
            if set(g.values()) & out_values:
                del xds.attrs["data_groups"][gname]
    else:
        for dv in group_out.values():
            assert dv not in dv_names, f"Data variable {dv} already exists in xds."
    return group_in, {**group_in, **group_out}
