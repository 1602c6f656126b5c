/* Alert sink for the oracle build of the reference sources: fatal, severe
 * and error alerts go to stderr when ORACLE_REF_VERBOSE is set, everything
 * else is dropped. */
#include <stdio.h>
#include <stdlib.h>
#include "difxmessage.h"

int difxMessageSendDifxAlert(const char *alertMessage, int severity)
{
	static int verbose = -1;
	if(verbose < 0)
		verbose = getenv("ORACLE_REF_VERBOSE") ? atoi(getenv("ORACLE_REF_VERBOSE")) : 0;
	if(verbose > 0 && severity <= (verbose > 1 ? DIFX_ALERT_LEVEL_DEBUG : DIFX_ALERT_LEVEL_ERROR))
		fprintf(stderr, "[ref alert %d] %s\n", severity, alertMessage);
	return 0;
}

int difxMessageSendDifxStatus3(int state, const char *message, double visMJD, int numdatastreams, float *weight,
                               double mjdStart, double mjdStop)
{
	(void)state; (void)message; (void)visMJD; (void)numdatastreams; (void)weight; (void)mjdStart; (void)mjdStop;
	return 0;
}

int difxMessageSendDifxDiagnosticBufferStatus(int threadid, int numelements, int startelement, int numactiveelements)
{
	(void)threadid; (void)numelements; (void)startelement; (void)numactiveelements;
	return 0;
}

int difxMessageSendDifxDiagnosticDataConsumed(long long bytes)
{
	(void)bytes;
	return 0;
}

int difxMessageSendDifxDiagnosticInputDatarate(double bytespersec)
{
	(void)bytespersec;
	return 0;
}
